"""Builds, trains and evaluates the learned steady-state initial guess on one
GPU (the chain4 family: 4-site chain, site energies U[0, 300] cm^-1,
couplings N(0, 60 cm^-1), 4 Drude baths lambda = 50 cm^-1, 1/gamma = 50 fs,
T = 300 K, K = 2, depth 8 = 125,970 nodes).

    python -m phi_b200.train_guess data  [--count 2048]   # steady states by BiCGSTAB(2)
    python -m phi_b200.train_guess train [--steps 4000]   # fit the MLP with the phi_nn_* kernels
    python -m phi_b200.train_guess eval  [--count 256]    # plain vs learned guess, same tolerance

Training draws use seeds TRAIN_SEED0 + k, evaluation draws EVAL_SEED0 + k
(disjoint).  Data and weights go to phi_b200/data/.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import capi, configs, learned
from .heom import Hierarchy

TRAIN_SEED0 = 10_000
EVAL_SEED0 = 1_000
DEPTH = 8
TOL = 1e-10
ELL = 2
MAX_STEPS = 40_000


def solve(p, rho0_guess=None, deflation: int = 0):
    """One steady-state solve (deflation: tiers of the deflation space, 0 =
    PHI's plain BiCGSTAB(2)); returns (rho_0, stats)."""
    p.fix_incompatible_combinations("bicgstab")
    with Hierarchy(p) as h:
        h.set_steady_deflation(deflation)
        st = h.steady_state(tol=TOL, ell=ELL, max_steps=MAX_STEPS, check=False, rho0_guess=rho0_guess)
        rho = h.rho0()
    return rho, st


def make_data(count: int, out: str = learned.DATASET, log=print):
    feats, targs, seeds, steps = [], [], [], []
    t0 = time.perf_counter()
    for k in range(count):
        p = configs.chain4(seed=TRAIN_SEED0 + k, depth=DEPTH)
        rho, st = solve(p)
        if st["status"] != capi.PHI_OK:
            continue  # only converged solves are training data
        feats.append(learned.chain_features(p))
        targs.append(learned.rho_to_coords(rho))  # rho_ss itself; train() subtracts the thermal state
        seeds.append(TRAIN_SEED0 + k)
        steps.append(st["steps"])
        if k % 64 == 0:
            log(f"data {k}/{count}: {st['steps']} steps, {time.perf_counter() - t0:.1f} s")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    np.savez(out, features=np.array(feats), targets=np.array(targs), seeds=np.array(seeds),
             steps=np.array(steps), depth=DEPTH, tol=TOL, ell=ELL)
    return {"solved": len(seeds), "requested": count, "seconds": time.perf_counter() - t0,
            "mean_steps": float(np.mean(steps)) if steps else None}


def train(steps: int, widths=(7, 128, 128, 16), data: str = learned.DATASET, out: str = learned.WEIGHTS):
    z = np.load(data)
    thermal = np.array([learned.rho_to_coords(learned.thermal_rho0(configs.chain4(seed=int(s), depth=DEPTH)))
                        for s in z["seeds"]])
    targets = z["targets"] - thermal
    m = learned.MLP(widths, seed=0)
    t0 = time.perf_counter()
    hist = m.fit(z["features"], targets, steps=steps)
    m.torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    m.save(out)
    pred = m.predict(z["features"]) + thermal
    err = np.abs(pred - z["targets"]).max(axis=1)
    return {"samples": int(len(z["seeds"])), "steps": steps, "seconds": sec, "loss_first": hist[0],
            "loss_last": hist[-1], "train_max_abs_err_median": float(np.median(err)),
            "thermal_max_abs_err_median": float(np.median(np.abs(thermal - z["targets"]).max(axis=1)))}


def evaluate(count: int, weights: str = learned.WEIGHTS, seed0: int = EVAL_SEED0, log=print):
    """Plain (rho_0 = I/N start), thermal-state start and learned-guess
    BiCGSTAB(2) on `count` held-out draws at the same tolerance, and the
    solver deflated by rho_0 and the first tier (from I/N and from the
    learned guess).  Wall time of the learned arm includes the network's
    inference."""
    model = learned.MLP.load(weights)
    rows = []
    for k in range(count):
        p = configs.chain4(seed=seed0 + k, depth=DEPTH)
        t0 = time.perf_counter()
        rho_a, sa = solve(p)
        ta = time.perf_counter() - t0
        t0 = time.perf_counter()
        guess = learned.predict_rho0(model, p)
        rho_b, sb = solve(p, rho0_guess=guess)
        tb = time.perf_counter() - t0
        thermal = learned.thermal_rho0(p)
        _, sc = solve(p, rho0_guess=thermal)
        t0 = time.perf_counter()
        rho_d, sd = solve(p, deflation=2)
        td = time.perf_counter() - t0
        _, sdl = solve(p, rho0_guess=guess, deflation=2)
        rows.append({"seed": seed0 + k, "plain_steps": sa["steps"], "learned_steps": sb["steps"],
                     "thermal_steps": sc["steps"],
                     "plain_device_s": sa["seconds"], "learned_device_s": sb["seconds"],
                     "plain_wall_s": ta, "learned_wall_s": tb,
                     "plain_ok": sa["status"] == capi.PHI_OK, "learned_ok": sb["status"] == capi.PHI_OK,
                     "thermal_ok": sc["status"] == capi.PHI_OK,
                     "deflated_steps": sd["steps"], "deflated_device_s": sd["seconds"], "deflated_wall_s": td,
                     "deflated_ok": sd["status"] == capi.PHI_OK and sd["deflated_tiers"] == 2,
                     "deflated_learned_steps": sdl["steps"], "deflated_learned_device_s": sdl["seconds"],
                     "deflated_learned_ok": sdl["status"] == capi.PHI_OK,
                     "deflated_rho0_diff": float(np.abs(rho_a - rho_d).max()),
                     "rho0_diff": float(np.abs(rho_a - rho_b).max()),
                     "guess_err": float(np.abs(guess - rho_a).max()),
                     "thermal_err": float(np.abs(thermal - rho_a).max()),
                     "identity_err": float(np.abs(np.eye(p.num_states) / p.num_states - rho_a).max())})
        if k % 32 == 0:
            log(f"eval {k}/{count}: plain {sa['steps']} learned {sb['steps']} deflated {sd['steps']}")
    ok = [r for r in rows if r["plain_ok"] and r["learned_ok"]]
    sum_plain = sum(r["plain_device_s"] for r in ok)
    sum_learned = sum(r["learned_device_s"] for r in ok)
    okd = [r for r in rows if r["plain_ok"] and r["deflated_ok"] and r["deflated_learned_ok"]]
    plain_d = sum(r["plain_device_s"] for r in okd)
    return {
        "deflated_failed": sum(1 for r in rows if not r["deflated_ok"]),
        "steps_deflated_mean": float(np.mean([r["deflated_steps"] for r in okd])) if okd else None,
        "steps_deflated_learned_mean": float(np.mean([r["deflated_learned_steps"] for r in okd])) if okd else None,
        "deflated_device_time_ratio": sum(r["deflated_device_s"] for r in okd) / plain_d if plain_d else None,
        "deflated_learned_device_time_ratio": (sum(r["deflated_learned_device_s"] for r in okd) / plain_d
                                               if plain_d else None),
        "deflated_wall_time_ratio": (sum(r["deflated_wall_s"] for r in okd) / sum(r["plain_wall_s"] for r in okd)
                                     if okd else None),
        "max_deflated_rho0_diff": max((r["deflated_rho0_diff"] for r in okd), default=None),
        "deflated_ms_per_solve": 1e3 * sum(r["deflated_device_s"] for r in okd) / len(okd) if okd else None,
        "plain_ms_per_solve": 1e3 * plain_d / len(okd) if okd else None,
        "draws": count, "both_converged": len(ok),
        "plain_failed": sum(1 for r in rows if not r["plain_ok"]),
        "learned_failed": sum(1 for r in rows if not r["learned_ok"]),
        "steps_plain_mean": float(np.mean([r["plain_steps"] for r in ok])) if ok else None,
        "steps_learned_mean": float(np.mean([r["learned_steps"] for r in ok])) if ok else None,
        "device_time_ratio": sum_learned / sum_plain if sum_plain else None,
        "wall_time_ratio": (sum(r["learned_wall_s"] for r in ok) / sum(r["plain_wall_s"] for r in ok)) if ok else None,
        "guess_err_median": float(np.median([r["guess_err"] for r in rows])) if rows else None,
        "thermal_err_median": float(np.median([r["thermal_err"] for r in rows])) if rows else None,
        "identity_err_median": float(np.median([r["identity_err"] for r in rows])) if rows else None,
        "steps_thermal_mean": float(np.mean([r["thermal_steps"] for r in ok])) if ok else None,
        "thermal_failed": sum(1 for r in rows if not r["thermal_ok"]),
        "max_rho0_diff": max((r["rho0_diff"] for r in ok), default=None),
        "rows": rows,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["data", "train", "eval"])
    ap.add_argument("--count", type=int, default=None)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--out", default=None, help="JSON result file")
    ap.add_argument("--data-path", default=learned.DATASET)
    ap.add_argument("--weights-path", default=learned.WEIGHTS)
    a = ap.parse_args()
    if a.what == "data":
        res = make_data(a.count or 2048, out=a.data_path)
    elif a.what == "train":
        res = train(a.steps, data=a.data_path, out=a.weights_path)
    else:
        res = evaluate(a.count or 256, weights=a.weights_path)
    text = json.dumps(res)
    if a.out:
        with open(a.out, "w") as f:
            f.write(text)
    print(json.dumps({k: v for k, v in res.items() if k != "rows"}))


if __name__ == "__main__":
    main()
