"""Benchmark: hierarchy-node Liouvillian applies per second of the RKF45
propagation of the 7-site Frenkel exciton hierarchy (N = 7, 7 Drude baths,
K = 1, depth L = 6: 38,760 nodes of 7x7 complex128; RKF45 tol 1e-6 to 1 ps).

One bench "step" is one attempted RKF45 step over the whole hierarchy: six
fused Liouvillian-apply + stage-combine kernels over all 38,760 nodes, the
error max-reduction and the device-side accept/step-size control.

The headline arithmetic is the mixed mode (complex64 stage inputs and
derivatives, FP32 Liouvillian, FP64 state / combines / error norm / step
control); the same run times the FP64 path and integrates the full 1 ps in
both to report the max-abs rho_0 error of the mixed mode against FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl phi_b200|reference]
                    [--precision fp64|mixed]

With N > 1 (torchrun, one rank per GPU) every rank integrates its own replica
of the hierarchy (the path has no exchange step): weak scaling, value = all
ranks' applies / max-over-ranks device time.  `--impl reference` times the
reference PHI build (oracle/_ref) on this host's cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "hierarchy-node applies/sec and RKF45 steps/sec at rho_0 err<=1e-6 vs FP64 GPU"
UNIT = "node-applies/s"
T_END = 1.0
DT0 = 0.001
TOL = 1e-6
MIN_DT = 1e-6


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=16)
    ap.add_argument("--impl", default="phi_b200", choices=["phi_b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="frenkel7",
                    choices=["frenkel7", "ring24", "batched", "steady", "spin_boson"],
                    help="frenkel7: the RKF45 headline (7-site exciton); ring24: 24-site ring RKF45; "
                         "batched: 512 uneven RK4 instances; steady: chain4 steady states, undeflated and "
                         "deflated, from I/N and from the learned initial guess; spin_boson: the 11-node "
                         "RK4 configuration")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--draws", type=int, default=32, help="steady workload: held-out draws")
    return ap.parse_args()


# RKF45 workloads: maker, t_end (ps), description.
RKF45_WORKLOADS = {
    "frenkel7": ("frenkel7", 1.0, "frenkel7_K1_L6: 7-site Frenkel exciton, 7 Drude baths, K=1, L=6, "
                                  "38760 nodes of 7x7, RKF45 tol 1e-6 to 1 ps"),
    "ring24": ("ring24", 0.5, "ring24_K0_L4: 24-site ring, 24 Drude baths, K=0, L=4, 20475 nodes of "
                              "24x24, RKF45 tol 1e-6 to 500 fs"),
}
WORKLOAD = "frenkel7"


def workload():
    from phi_b200 import configs
    p = getattr(configs, RKF45_WORKLOADS[WORKLOAD][0])()
    p.fix_incompatible_combinations("rkf45")
    return p


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def wait_first_sample(self, timeout=5.0):
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.05)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model() -> str:
    """CPU model name of this host (from /proc/cpuinfo) and its logical CPU count."""
    name = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                name = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{name} ({os.cpu_count()} logical CPUs)"


def reference_fixture(workload_name):
    """rho_0 of the reference build for the full-size RKF45 workload (the
    committed fixture tests/golden/ref_fullsize.json), or None."""
    import numpy as np
    path = os.path.join(ROOT, "tests", "golden", "ref_fullsize.json")
    if not os.path.exists(path):
        return None
    fixture_id = {"frenkel7": "frenkel7_L6/rkf45", "ring24": "ring24_L4/rkf45"}.get(workload_name)
    for c in json.load(open(path))["cases"]:
        if c["id"] == fixture_id and c.get("rho0_colmajor"):
            v = np.array(c["rho0_colmajor"])
            n = int(round(len(v) ** 0.5))
            rho = (v[:, 0] + 1j * v[:, 1]).reshape(n, n).T
            return rho, c
    return None


def cpu_baseline_port(p, seconds_budget=10.0):
    """The oracle (C restatement, one core) on a bounded sample: Liouvillian
    applies over the full hierarchy until seconds_budget of CPU work (at most
    400 applies)."""
    import numpy as np
    from oracle import oracle as O
    o = O.Oracle(p)
    s = o.initial_state()
    rng = np.random.default_rng(0)
    s = s + 1e-3 * rng.normal(size=s.size)
    n_apply = 0
    t0 = time.perf_counter()
    while True:
        o.apply(s)
        n_apply += 1
        if time.perf_counter() - t0 >= seconds_budget or n_apply >= 400:
            break
    dt = time.perf_counter() - t0
    return {"value": n_apply * o.M / dt, "unit": UNIT, "cores": 1, "kind": "port", "cpu": cpu_model(),
            "sample": f"{n_apply} Liouvillian applies over the {o.M}-node hierarchy "
                      f"({dt:.1f} s, single-thread C restatement)"}


def run_reference_arm(args):
    """Times the reference PHI build (oracle/_ref/ref_driver: PhiParameters ->
    HierarchyIntegrator::Launch, unchanged) with all host threads on the same
    workload.  The figure is PHI's own integration timer: the output file's
    "#Total integration time" (whole seconds, hierarchy_integrator.cc:2527-2538)
    over its "#Total number of integration steps", from a run sized to
    integrate for about 20 s, so the O(M^2) setup PHI does before it is
    excluded and the timer's 1 s resolution costs at most 5 %."""
    from oracle import oracle as O
    from phi_b200 import configs
    p = workload()
    threads = os.cpu_count() or 1
    res = {"impl": "reference", "metric": METRIC, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
           "config": {"workload": RKF45_WORKLOADS[WORKLOAD][2], "seed": p.seed, "threads": threads}}
    if not O.ref_available():
        res["unavailable"] = "reference build oracle/_ref/ref_driver not present"
        return res

    def run(t_end):
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "phi.out")
            prm = os.path.join(d, "in.prm")
            rho_f = os.path.join(d, "rho.txt")
            with open(prm, "w") as f:
                f.write(O.param_file_text(p, timestep=DT0, t_end=t_end, output_file=out)
                        .replace("verbose=-2", "verbose=0"))
            subprocess.run([O.REF_DRIVER, "run", prm, "rkf45", str(threads), rho_f], check=True,
                           timeout=900, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            steps = secs = None
            for ln in open(out):
                if ln.startswith("#Total number of integration steps"):
                    steps = int(ln.split("=")[1])
                if ln.startswith("#Total integration time"):
                    secs = 60.0 * float(ln.split("=")[1].split()[0])
            return steps, secs

    try:
        t_end = 0.002 + 0.001 * max(2, min(args.steps, 8))
        steps, secs = run(t_end)
        for _ in range(3):  # lengthen the run until PHI's timer reads about 20 s
            if steps is None or secs is None or secs >= 15:
                break
            t_end = min(T_END, t_end * (20.0 / max(secs, 1.0)))
            steps, secs = run(t_end)
            if t_end >= T_END:
                break
    except subprocess.TimeoutExpired:
        res["unavailable"] = "reference RKF45 run timed out (its accept test races with the writer thread)"
        return res
    if not steps or not secs:
        res["unavailable"] = f"reference run too short to time: {steps} steps in {secs} s"
        return res
    M = configs.hierarchy_nodes(int(p.num_bath_couplings) * int(p.num_matsubara_terms),
                                int(p.hierarchy_truncation_level) - 1)
    per_step = secs / steps
    value = 6 * M / per_step
    res.update({"value": value, "ms_per_step": per_step * 1e3,
                "rkf45_steps_per_s": 1.0 / per_step,
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                                 "cpu": cpu_model(),
                                 "sample": f"{steps} RKF45 steps to t = {t_end:.4g} ps in {secs:.0f} s by PHI's "
                                           f"own integration timer, {threads} threads"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    return res


def run_spin_boson(args):
    """The spin-boson configuration (one Drude bath on sigma_z, DiagonalBath,
    K = 0, L = 10: 11 nodes of 2x2; RK4 dt = 1 fs, 2000 steps = 2 ps, rho_0
    every 10 fs).  The hierarchy is 44 complex numbers, so the run is bound
    by latency, not by HBM or the SMs: the device runs it whole in one CTA
    (heom_small.cu), one launch per 4096 steps.  A step is one RK4 step (4
    Liouvillian applies over the hierarchy); value = node-applies/s of the
    device-timed steps; e2e = the whole job through the C ABI from host
    arrays (create, 2000 steps with the trajectory rows, read-back, destroy).
    The reference arm runs the reference build with one thread, its fastest
    setting for this size (the thread barriers of more threads cost more
    than the 44 elements of work per stage)."""
    import numpy as np
    from phi_b200 import configs
    p = configs.spin_boson()
    dt, K = 0.001, args.steps if args.steps > 0 else 2000
    M = configs.hierarchy_nodes(1, 10)
    base = {"metric": "hierarchy-node applies/sec (RK4, spin-boson)", "unit": UNIT, "n_gpus": 1,
            "steps": K, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic (spin-boson, fixed parameters)",
            "config": {"workload": "spin_boson_L10 (11 nodes of 2x2, DiagonalBath, RK4 dt 1 fs)", "nodes": M,
                       "parallelism": "single instance"}}
    if args.impl == "reference":
        from oracle import oracle as O
        res = dict(base, impl="reference")
        if not O.ref_available():
            res["unavailable"] = "reference build oracle/_ref/ref_driver not present"
            print(json.dumps(res), flush=True)
            return

        def wall(t_end):
            best = float("inf")
            for _ in range(3):
                t0 = time.perf_counter()
                O.run_reference(p, "rk4", 1, timeout=300, timestep=dt, t_end=t_end)
                best = min(best, time.perf_counter() - t0)
            return best
        # Per step from the difference of two run lengths (process start and
        # setup cancel).
        long_steps, short_steps = 20 * K, 2 * K
        per_step = (wall(long_steps * dt) - wall(short_steps * dt)) / (long_steps - short_steps)
        value = 4 * M / per_step
        res.update({"value": value, "ms_per_step": per_step * 1e3,
                    "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                                     "cpu": cpu_model(),
                                     "sample": f"reference build, RK4 runs of {long_steps} and {short_steps} steps "
                                               f"(wall time difference, best of 3), 1 thread"},
                    "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        print(json.dumps(res), flush=True)
        return

    import torch
    from phi_b200 import capi
    from phi_b200.heom import Hierarchy
    h = Hierarchy(p)
    stream = torch.cuda.ExternalStream(h.stream_handle())
    h.rk4(dt, max(args.warmup, 3) * dt)
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    sampler.wait_first_sample()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h.rk4(dt, h.time + K * dt * (1 - 1e-9))
    e1.record(stream)
    e1.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    value = 4 * M * K / (ms / 1e3)
    h.close()
    # e2e: the user job of the configuration, warm process, second run reported.
    rows = 200
    for _ in range(2):
        t0 = time.perf_counter()
        h2 = Hierarchy(p)
        h2.rk4(dt, K * dt, output_min_step=0.01, capacity=rows)
        rho0 = h2.rho0()
        h2.close()
        e2e_s = time.perf_counter() - t0
    from oracle import oracle as O
    o = O.Oracle(p)
    s_o, *_ = o.rk4(o.initial_state(), dt, K * dt)
    err = float(np.abs(rho0 - o.rho0(s_o)).max())
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < 5.0:
        o.rk4(o.initial_state(), dt, K * dt)
        reps += 1
    cpu_s = (time.perf_counter() - t0) / reps
    out = dict(base)
    out.update({"value": value, "ms_per_step": ms / K,
                "roofline": None,
                "roofline_note": "latency-bound: 44 complex elements live in one CTA's shared memory for the "
                                 "whole run (no HBM traffic per step); the bound is the per-stage barrier and "
                                 "shared-memory latency",
                "rho0_err_vs_oracle": err,
                "e2e": {"value": 4 * M * K / e2e_s, "unit": UNIT, "seconds": e2e_s,
                        "h2d_bytes_per_step": (2 * 4 + 2 * 4 + 2 + 2) * 8 / K,
                        "d2h_bytes_per_step": (rows * 4 * 16 + 4 * 16) / K},
                "cpu_baseline": {"value": 4 * M * K / cpu_s, "unit": UNIT, "cores": 1, "kind": "port",
                                 "cpu": cpu_model(),
                                 "sample": f"the oracle's C restatement, the whole {K}-step run x {reps}"},
                "gpu_launches": (K + 4095) // 4096,
                "clocks": clocks})
    print(json.dumps(out), flush=True)


def run_steps(h, steps, fresh):
    """Exactly `steps` attempted RKF45 steps of the 1 ps propagation; when a
    propagation reaches t_end it restarts from rho(0) on the device
    (phi_gpu_reset).  Returns (steps, propagations finished, advance calls)."""
    done = finished = calls = 0
    dt0 = DT0 if fresh else -1.0
    while done < steps:
        st = h.rkf45_advance(dt0, T_END, TOL, MIN_DT, steps - done)
        calls += 1
        done += int(st["steps"])
        dt0 = -1.0
        if st["final_time"] >= T_END:
            h.reset(0.0)
            finished += 1
            dt0 = DT0
    return done, finished, calls


def batch_step_bytes(problems, mixed):
    """Algorithmic bytes of one fused RK4 step over all instances.  FP64: 16
    complex128 state-size transfers (stage 0 reads y, writes X1 and acc;
    stages 1-2 read X, y, acc and write X', acc; stage 3 reads X3, acc and
    writes y).  Mixed: 10 complex128 (y, acc) and 8 complex64 (X, y32)
    transfers, complex64 nodes padded to an even element count."""
    total = 0
    for p in problems:
        E = p.num_states ** 2
        EP = E + (E & 1)
        total += p.nodes * (10 * E * 16 + 8 * EP * 8 if mixed else 16 * E * 16)
    return total


def run_batched(args):
    """Batched uneven instances: every RK4 stage of all instances in one
    persistent launch; value = node-applies/s = 4 * steps * total nodes /
    device time.  Also times the other arithmetic and reports the max-abs
    rho_0 difference between the two after the same steps."""
    import numpy as np
    import torch
    from phi_b200 import capi, configs
    from phi_b200.heom import Batch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    problems_all = configs.batched(seed=3, count=args.batch_count)
    # Shards: a size-balanced greedy split of the instances over the ranks
    # (no collective on the data path).
    from phi_b200.shard import balanced_shards
    shards = balanced_shards([p.nodes * p.num_states ** 2 for p in problems_all], world)
    problems = [problems_all[i] for i in shards[rank]]
    dt = 0.0005
    prec = capi.PHI_PREC_MIXED if args.precision == "mixed" else capi.PHI_PREC_FP64
    results = {}
    rho = {}
    clocks = None
    for pr in ([prec, capi.PHI_PREC_FP64] if prec == capi.PHI_PREC_MIXED else [prec]):
        t0 = time.perf_counter()
        b = Batch(problems, precision=pr, device=local_rank)
        create_s = time.perf_counter() - t0
        sched = b.autotune()
        b.rk4(dt, args.warmup)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        sampler = None
        if pr == prec:
            sampler = ClockSampler(local_rank)
            sampler.start()
            sampler.wait_first_sample()
        st = b.rk4(dt, args.steps)
        if sampler:
            clocks = sampler.stop()
        sec = st["seconds"]
        if dist:
            t = torch.tensor([sec], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            sec = float(t.item())
            na = torch.tensor([st["node_applies"]], device="cuda", dtype=torch.int64)
            dist.all_reduce(na, op=dist.ReduceOp.SUM)
            applies = int(na.item())
        else:
            applies = st["node_applies"]
        rho[pr] = [b[i].rho0() for i in range(b.count)]
        results[pr] = {"seconds": sec, "applies": applies, "schedule": sched, "create_s": create_s,
                       "launches": st["launches"], "ms_per_step": sec * 1e3 / args.steps}
        b.close()
        torch.cuda.synchronize()
    r = results[prec]
    rho_err = None
    if prec == capi.PHI_PREC_MIXED:
        rho_err = max(float(np.abs(a - c).max()) for a, c in zip(rho[prec], rho[capi.PHI_PREC_FP64]))
        if dist:
            t = torch.tensor([rho_err], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            rho_err = float(t.item())
    if rank == 0:
        peak, peak_kind = peaks()
        step_bytes = batch_step_bytes(problems, prec == capi.PHI_PREC_MIXED)
        achieved = step_bytes / (r["ms_per_step"] / 1e3) / 1e9
        summ = configs.batch_summary(problems_all)
        out = {
            "metric": METRIC, "value": r["applies"] / r["seconds"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
            "dtype": "c128" if prec == capi.PHI_PREC_FP64 else "c64 stages (fp32 Liouvillian) + c128 state",
            "data": "synthetic (seeded batched instances, numpy default_rng seed 3)",
            "config": {"workload": f"batched: {args.batch_count} uneven chain instances, N in {{2..16}}, "
                                   "K in {0,1}, L 4-10 under a 256 MiB/instance budget, RK4 dt 0.5 fs",
                       "precision": args.precision, "parallelism": f"instance shards x{world}",
                       "l2": "working set > 20 GB >> 126 MB L2", **summ},
            "rho0_err_vs_fp64": rho_err,
            "meets_1e-6": None if rho_err is None else rho_err <= 1e-6,
            "schedule": r["schedule"], "create_seconds": r["create_s"],
            "other_precision": None if len(results) == 1 else {
                "precision": "fp64", "ms_per_step": results[capi.PHI_PREC_FP64]["ms_per_step"],
                "value": results[capi.PHI_PREC_FP64]["applies"] / results[capi.PHI_PREC_FP64]["seconds"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "heom_tile_batch_kernel x4 (one RK4 step of every instance)",
                         "algorithmic_bytes_per_step": step_bytes, "peak_kind": peak_kind},
            "gpu_launches": r["launches"],
            "clocks": clocks,
        }
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_steady(args):
    """chain4 steady states (4-site chain, K=2, depth 8: 125,970 nodes of
    4x4): BiCGSTAB(2) to ||r||/||b|| <= 1e-10 from I/N, from the thermal
    state and from the learned rho_0, undeflated (PHI's solver) and deflated
    by the ADOs of tiers 0-1 (the library's default), on `--draws` held-out
    draws; value = node-applies/s of the undeflated solves (2 applies per
    BiCG step), ms_per_step = device time of one default (deflated) solve."""
    import numpy as np
    import torch
    from phi_b200 import train_guess
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    res = train_guess.evaluate(args.draws)
    rows = [r for r in res["rows"] if r["plain_ok"] and r["learned_ok"]]
    M = 125970
    plain_s = sum(r["plain_device_s"] for r in rows)
    plain_steps = sum(r["plain_steps"] for r in rows)
    value = 2 * M * plain_steps / plain_s if plain_s else None
    out = {"metric": "steady-state solve: node-applies/s and wall time to ||r||/||b|| <= 1e-10",
           "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.draws, "warmup": 0,
           "ms_per_step": res["deflated_ms_per_solve"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "c128", "data": "synthetic (chain4 family, seeds 1000+)",
           "config": {"workload": "chain4_K2_L8: 4-site chain, 4 Drude baths, K=2, L=8, 125970 nodes of 4x4; "
                                  "BiCGSTAB(2), relative residual 1e-10", "draws": args.draws},
           "undeflated_ms_per_solve": res["plain_ms_per_solve"],
           "solver_arms": {k: v for k, v in res.items() if k != "rows"},
           "gpu_launches": None}
    print(json.dumps(out), flush=True)


def dgemm_peak_tflops(n: int = 8192, reps: int = 5) -> float:
    """Measured FP64 matrix-multiply rate of this GPU (cuBLAS DGEMM through
    torch.matmul on float64), 2 n^3 flops per product, best of reps."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = torch.matmul(a, b)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def main():
    global WORKLOAD, T_END
    args = parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference" and args.workload in ("batched", "steady"):
        if int(os.environ.get("RANK", "0")) == 0:
            why = ("the reference's steady-state solvers crash or return NaN on in-scope inputs"
                   if args.workload == "steady" else
                   "not timed for this workload: the reference integrates one problem per process "
                   "(its CPU path is timed on the frenkel7 and ring24 workloads)")
            print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
        return
    if args.workload == "spin_boson":
        if int(os.environ.get("RANK", "0")) == 0:
            run_spin_boson(args)
        return
    if args.workload == "batched":
        run_batched(args)
        return
    if args.workload == "steady":
        if int(os.environ.get("RANK", "0")) == 0:
            run_steady(args)
        return
    WORKLOAD = args.workload
    T_END = RKF45_WORKLOADS[WORKLOAD][1]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference_arm(args)), flush=True)
        return

    import torch
    import numpy as np
    from phi_b200 import capi
    from phi_b200.heom import Hierarchy

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    prec = capi.PHI_PREC_MIXED if args.precision == "mixed" else capi.PHI_PREC_FP64
    p = workload()
    N = p.num_states

    # ---- device-resident throughput (value) ----
    h = Hierarchy(p, precision=prec, device=local_rank)
    M = h.num_nodes
    T_terms = h.num_terms
    tile_sched = h.tile_schedule()
    stream = torch.cuda.ExternalStream(h.stream_handle(), device=local_rank)
    run_steps(h, args.warmup, True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    sampler.wait_first_sample()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    steps_done, propagations, advance_calls = run_steps(h, args.steps, False)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    t_max = ms
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
        sd = torch.tensor([steps_done], device="cuda")
        dist.all_reduce(sd, op=dist.ReduceOp.SUM)
        total_steps = int(sd.item())
    else:
        total_steps = steps_done
    applies = 6 * M * total_steps
    value = applies / (t_max / 1e3)
    ms_per_step = t_max / max(steps_done, 1)

    # ---- dominant kernel in isolation: one apply launch over all nodes ----
    E = N * N
    EPX = (E + (E & 1)) if prec == capi.PHI_PREC_MIXED else E
    if prec == capi.PHI_PREC_MIXED:
        x = torch.randn(M * EPX * 2, dtype=torch.float32, device="cuda")
    else:
        x = torch.randn(M * E * 2, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    reps = 20
    with torch.cuda.stream(stream):
        for _ in range(3):
            capi.check(h.lib.phi_gpu_apply_device(h.ctx, x.data_ptr(), y.data_ptr(), stream.cuda_stream), h.ctx)
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    for _ in range(reps):
        capi.check(h.lib.phi_gpu_apply_device(h.ctx, x.data_ptr(), y.data_ptr(), stream.cuda_stream), h.ctx)
    eb.record(stream)
    eb.synchronize()
    apply_ms = ea.elapsed_time(eb) / reps
    h.close()

    # ---- end to end through the C ABI with host buffers ----
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    # The user job: build the hierarchy on the device from host arrays, run the
    # whole 1 ps RKF45 propagation, read rho_0 back, tear down.  Run twice in
    # this warm process; the second run is reported.
    for _ in range(2):
        t0 = time.perf_counter()
        h2 = Hierarchy(p, precision=prec, device=local_rank)
        st2 = h2.rkf45(DT0, T_END, TOL, MIN_DT)
        rho0 = h2.rho0()
        h2.close()
        e2e_s = time.perf_counter() - t0
    e2e_steps = int(st2["steps"])
    e2e_value = 6 * M * e2e_steps / e2e_s
    if dist:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_value = 6 * M * e2e_steps * world / float(t.item())
    h2d = (2 * E + 2 * E + 2 * int(p.num_bath_couplings)) * 8  # H, rho(0), gamma, lambda
    d2h = 2 * E * 8 + ((e2e_steps + 15) // 16 + 1) * 320  # rho_0 + control-block polls

    # ---- the other arithmetic, and the full 1 ps rho_0 error of mixed vs FP64 ----
    other = capi.PHI_PREC_FP64 if prec == capi.PHI_PREC_MIXED else capi.PHI_PREC_MIXED
    ho = Hierarchy(p, precision=other, device=local_rank)
    so = torch.cuda.ExternalStream(ho.stream_handle(), device=local_rank)
    run_steps(ho, args.warmup, True)
    torch.cuda.synchronize()
    e0o, e1o = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0o.record(so)
    other_steps, _, _ = run_steps(ho, args.steps, False)
    e1o.record(so)
    e1o.synchronize()
    other_ms_per_step = e0o.elapsed_time(e1o) / max(other_steps, 1)
    ho.close()
    rho_full = {}
    for pr in (capi.PHI_PREC_FP64, capi.PHI_PREC_MIXED):
        hf = Hierarchy(p, precision=pr, device=local_rank)
        stf = hf.rkf45(DT0, T_END, TOL, MIN_DT)
        rho_full[pr] = (hf.rho0(), stf)
        hf.close()
    rho_err = float(np.abs(rho_full[capi.PHI_PREC_MIXED][0] - rho_full[capi.PHI_PREC_FP64][0]).max())
    # Against the reference build's own FP64 rho_0 of the same full run.
    vs_ref = None
    fx = reference_fixture(WORKLOAD)
    if fx is not None:
        rho_ref, meta = fx
        vs_ref = {"fp64": float(np.abs(rho_full[capi.PHI_PREC_FP64][0] - rho_ref).max()),
                  "mixed": float(np.abs(rho_full[capi.PHI_PREC_MIXED][0] - rho_ref).max()),
                  "reference_steps": meta["steps"], "reference_accepted": meta["accepted_steps"],
                  "source": "tests/golden/ref_fullsize.json (reference build, %.17g)"}

    if rank == 0:
        peak, peak_kind = peaks()
        S = M * E * 16
        EP = E + (E & 1)
        # Algorithmic bytes of one fused RKF45 step: FP64 touches
        # 36 complex128 state-size arrays; mixed touches 2 complex128 (stage 5
        # reads y and writes y5) and 35 complex64 ones (stage inputs, k, the
        # complex64 copy y32 that stages 1-4 combine from and stage 5 writes).
        step_bytes = 36 * S if prec == capi.PHI_PREC_FP64 else M * (2 * E * 16 + 35 * EP * 8)
        achieved = step_bytes / (ms_per_step / 1e3) / 1e9
        apply_bytes = 2 * S if prec == capi.PHI_PREC_FP64 else 2 * M * EPX * 8
        apply_gbs = apply_bytes / (apply_ms / 1e3) / 1e9
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath) and WORKLOAD == "frenkel7" and prec == capi.PHI_PREC_MIXED:
            try:
                traffic = json.load(open(tpath)).get("rkf45_step_dram_bytes")
            except Exception:
                traffic = None
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128" if prec == capi.PHI_PREC_FP64 else "c64 stages (fp32 Liouvillian) + c128 state/norms",
            "data": f"synthetic (seeded {WORKLOAD}, numpy default_rng seed {p.seed})",
            "config": {"workload": RKF45_WORKLOADS[WORKLOAD][2],
                       "nodes": M, "num_states": N, "terms": T_terms,
                       "precision": args.precision, "parallelism": f"replicas x{world}",
                       "l2": f"working set 9 x {M * E * 16 / 1e6:.1f} MB state buffers = "
                             f"{9 * M * E * 16 / 1e6:.0f} MB > 126 MB L2"},
            "rkf45_steps_per_s": total_steps / (t_max / 1e3),
            "tile_schedule": tile_sched,
            "rho0_err_vs_fp64": rho_err,
            "rho0_err_vs_reference": vs_ref,
            "meets_1e-6": rho_err <= 1e-6 and (vs_ref is None or vs_ref["mixed"] <= 1e-6),
            "full_run": {"t_end_ps": T_END,
                         "fp64_steps": int(rho_full[capi.PHI_PREC_FP64][1]["steps"]),
                         "fp64_accepted": int(rho_full[capi.PHI_PREC_FP64][1]["accepted"]),
                         "mixed_steps": int(rho_full[capi.PHI_PREC_MIXED][1]["steps"]),
                         "mixed_accepted": int(rho_full[capi.PHI_PREC_MIXED][1]["accepted"])},
            "other_precision": {"precision": "fp64" if other == capi.PHI_PREC_FP64 else "mixed",
                                "ms_per_step": other_ms_per_step,
                                "value": 6 * M / (other_ms_per_step / 1e3)},
            "speedup_vs_fp64": (other_ms_per_step / ms_per_step) if other == capi.PHI_PREC_FP64 else
                               (ms_per_step / other_ms_per_step),
            "steps_timed": steps_done,
            "propagations_completed_in_timed_region": propagations,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "heom_tile_kernel x6 + rkf45_control_kernel (one RKF45 step)",
                         "algorithmic_bytes_per_step": step_bytes, "peak_kind": peak_kind},
            "apply_kernel": {"ms": apply_ms, "algorithmic_bytes": apply_bytes, "achieved_gbs": apply_gbs,
                             "frac": apply_gbs / peak, "node_applies_per_s": M / (apply_ms / 1e3)},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / max(e2e_steps, 1),
                    "d2h_bytes_per_step": d2h / max(e2e_steps, 1),
                    "what": "create (hierarchy built on device) + full 1 ps RKF45 + rho_0 read-back + "
                            "destroy, host wall clock through the C ABI (second of two runs)", "rho0_trace": float(np.trace(rho0).real)},
            # six stage kernels + the control kernel per attempted step, and the
            # complex64 copy of y each advance call starts with (mixed)
            "gpu_launches": 7 * steps_done + (advance_calls if prec == capi.PHI_PREC_MIXED else 0),
            "clocks": clocks,
        }
        if WORKLOAD == "ring24":
            # N = 24 sits near the FP64 ridge: the FP64 path's compute
            # roofline, 8 N^3 flops per node apply (one complex N x N
            # product), against the measured FP64 GEMM rate of this GPU.
            fp64_ms = ms_per_step if prec == capi.PHI_PREC_FP64 else other_ms_per_step
            fp64_applies = 6 * M / (fp64_ms / 1e3)
            flops = 8 * N ** 3
            dpeak = dgemm_peak_tflops()
            ach = fp64_applies * flops / 1e12
            out["fp64_compute_roofline"] = {
                "achieved_tflops": ach, "peak_tflops": dpeak, "frac": ach / dpeak,
                "flops_per_apply": flops, "node_applies_per_s": fp64_applies,
                "peak_kind": "measured: cuBLAS DGEMM 8192^3 (torch.matmul float64), best of 5"}
        if not args.no_cpu_baseline and world == 1:
            out["cpu_baseline"] = cpu_baseline_port(p)
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
