// heom_hierarchy.cu -- hierarchy construction on the device.
//
// Replaces Hierarchy::ConstructI (hierarchy.cc:45-155) and the neighbour
// search of HierarchyIntegrator::LinkHierarchyNodes
// (hierarchy_integrator.cc:1204-1338), which PHI does with std::map lookups.
//
// PHI's order: tier l is built from tier l-1 (C nodes, ids f..f+C-1) by
// visiting candidates q = k*C + n for k in [0,T), n in [0,C):
//     cand(q) = node(f + n) + e_{(n + k) mod T}
// and appending each multi-index the first time it is seen.  So the tier-l
// ids are the distinct candidates ordered by their smallest q.
//
// On the device every multi-index of tier l is named by its colex rank among
// the compositions of l into T parts (stars and bars: bar j sits at
// p_j = n_0 + ... + n_j + j, rank = sum_j C(p_j, j+1)).  Per tier:
//   1. first_q[rank(cand(q))] = min q          (atomicMin)
//   2. keep[q] = first_q[rank(cand(q))] == q   (first occurrence)
//   3. exclusive scan of keep -> position in the tier
//   4. scatter multi-indices, rank_to_id[rank] = id
// Neighbour ids then follow from ranks: rank(n +- e_t) differs from rank(n)
// only in the bars j >= t, so all T of them come from one prefix/suffix pass.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "heom_device.cuh"
#include "heom_internal.h"

namespace phi {
namespace {

constexpr int kScanBlock = 512;

// Binomial table C(a, b) for a <= amax, b <= bmax, row-major (bmax + 1) wide.
struct Binom {
  const unsigned long long *tab;
  int width;
  __device__ __forceinline__ unsigned long long operator()(int a, int b) const {
    if (b < 0 || a < b || a < 0) return 0ull;
    return tab[a * width + b];
  }
};

// Candidate q of tier `level`: multi-index of node (prev_first + n) plus e_{(n+k) mod T}.
__device__ __forceinline__ unsigned long long candidate_rank(const uint8_t *mi, int T,
                                                             long long prev_first,
                                                             long long C, long long q,
                                                             Binom binom, int *bump) {
  const long long k = q / C;
  const long long n = q - k * C;
  const int t = (int)((n + k) % T);
  const uint8_t *v = mi + (prev_first + n) * T;
  unsigned long long r = 0;
  int s = 0;
  for (int j = 0; j + 1 < T; ++j) {
    s += v[j] + (j == t ? 1 : 0);
    r += binom(s + j, j + 1);
  }
  *bump = t;
  return r;
}

__global__ void init_first_q_kernel(unsigned long long *first_q, long long count) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; i < count; i += (long long)gridDim.x * blockDim.x) first_q[i] = ~0ull;
}

__global__ void first_occurrence_kernel(const uint8_t *mi, int T, long long prev_first,
                                        long long C, long long num_cand, Binom binom,
                                        unsigned long long *first_q) {
  long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; q < num_cand; q += (long long)gridDim.x * blockDim.x) {
    int t;
    unsigned long long r = candidate_rank(mi, T, prev_first, C, q, binom, &t);
    atomicMin(first_q + r, (unsigned long long)q);
  }
}

// keep[q] and per-block sums of keep.
__global__ void keep_flags_kernel(const uint8_t *mi, int T, long long prev_first, long long C,
                                  long long num_cand, Binom binom,
                                  const unsigned long long *first_q, uint8_t *keep,
                                  long long *block_sums) {
  __shared__ int warp_sums[kScanBlock / 32];
  long long q = blockIdx.x * (long long)kScanBlock + threadIdx.x;
  int flag = 0;
  if (q < num_cand) {
    int t;
    unsigned long long r = candidate_rank(mi, T, prev_first, C, q, binom, &t);
    flag = first_q[r] == (unsigned long long)q;
    keep[q] = (uint8_t)flag;
  }
  int w = __popc(__ballot_sync(0xffffffffu, flag));
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = w;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int i = 0; i < kScanBlock / 32; ++i) s += warp_sums[i];
    block_sums[blockIdx.x] = s;
  }
}

// Exclusive scan of the block sums (single CTA, serial chunks).
__global__ void scan_block_sums_kernel(long long *block_sums, long long nblocks,
                                       long long *total) {
  __shared__ long long chunk[1024];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (long long base = 0; base < nblocks; base += 1024) {
    long long i = base + threadIdx.x;
    long long v = i < nblocks ? block_sums[i] : 0;
    chunk[threadIdx.x] = v;
    __syncthreads();
    // Hillis-Steele inclusive scan in shared memory.
    for (int off = 1; off < 1024; off <<= 1) {
      long long add = threadIdx.x >= (unsigned)off ? chunk[threadIdx.x - off] : 0;
      __syncthreads();
      chunk[threadIdx.x] += add;
      __syncthreads();
    }
    if (i < nblocks) block_sums[i] = carry + chunk[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += chunk[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

// Scatter the kept candidates into tier order.
__global__ void scatter_tier_kernel(uint8_t *mi, int T, long long prev_first, long long C,
                                    long long num_cand, long long tier_first, long long tier_count,
                                    Binom binom, const uint8_t *keep,
                                    const long long *block_offsets, int32_t *rank_to_id,
                                    int *bad) {
  __shared__ int warp_prefix[kScanBlock / 32];
  long long q = blockIdx.x * (long long)kScanBlock + threadIdx.x;
  int flag = q < num_cand ? keep[q] : 0;
  unsigned ballot = __ballot_sync(0xffffffffu, flag);
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_prefix[warp] = __popc(ballot);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int i = 0; i < kScanBlock / 32; ++i) {
      int v = warp_prefix[i];
      warp_prefix[i] = s;
      s += v;
    }
  }
  __syncthreads();
  if (flag) {
    long long pos = block_offsets[blockIdx.x] + warp_prefix[warp] +
                    __popc(ballot & ((1u << lane) - 1u));
    long long id = tier_first + pos;
    int t;
    unsigned long long r = candidate_rank(mi, T, prev_first, C, q, binom, &t);
    if (pos < 0 || pos >= tier_count || r >= (unsigned long long)tier_count) {
      atomicExch(bad, 1);  // never write outside the tier
      return;
    }
    const long long k = q / C;
    const long long n = q - k * C;
    const uint8_t *src = mi + (prev_first + n) * T;
    uint8_t *dst = mi + id * T;
    for (int j = 0; j < T; ++j) dst[j] = src[j] + (j == t ? 1 : 0);
    rank_to_id[r] = (int32_t)id;
  }
}

// next/prev ids of every node from ranks (see file comment).
__global__ void link_kernel(const uint8_t *mi, int T, int L, long long M, Binom binom,
                            const long long *tier_first, const int32_t *rank_to_id,
                            int32_t *next, int32_t *prev, int *bad) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; i < M; i += (long long)gridDim.x * blockDim.x) {
    const uint8_t *v = mi + i * T;
    unsigned long long base[kMaxTerms], up[kMaxTerms], dn[kMaxTerms];
    int s = 0, tier = 0;
    for (int j = 0; j < T; ++j) tier += v[j];
    for (int j = 0; j + 1 < T; ++j) {
      s += v[j];
      const int p = s + j;
      base[j] = binom(p, j + 1);
      up[j] = binom(p + 1, j + 1);
      dn[j] = binom(p - 1, j + 1);
    }
    // Suffix sums of up/dn over j >= t (bars j in [t, T-2]).
    unsigned long long su = 0, sd = 0;
    unsigned long long suf_up[kMaxTerms], suf_dn[kMaxTerms];
    for (int j = T - 1; j >= 0; --j) {
      if (j + 1 < T) {
        su += up[j];
        sd += dn[j];
      }
      suf_up[j] = su;
      suf_dn[j] = sd;
    }
    unsigned long long pre = 0;
    for (int t = 0; t < T; ++t) {
      int32_t nx = -1, pv = -1;
      if (tier > L) {
        atomicExch(bad, 1);
        break;
      }
      if (tier < L) {
        const unsigned long long r = pre + suf_up[t];
        const long long cnt = tier_first[tier + 2] - tier_first[tier + 1];
        if (r < (unsigned long long)cnt) nx = rank_to_id[tier_first[tier + 1] + r];
        else atomicExch(bad, 1);
      }
      if (v[t] > 0 && tier > 0) {
        const unsigned long long r = pre + suf_dn[t];
        const long long cnt = tier_first[tier] - tier_first[tier - 1];
        if (r < (unsigned long long)cnt) pv = rank_to_id[tier_first[tier - 1] + r];
        else atomicExch(bad, 1);
      }
      next[i * T + t] = nx;
      prev[i * T + t] = pv;
      if (t + 1 < T) pre += base[t];
    }
  }
}

int blocks_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 64) b = 148 * 64;
  return (int)b;
}

}  // namespace

// Host driver.  Counts per tier come from the binomial table: the number of
// compositions of l into T parts is C(l + T - 1, T - 1).
int build_hierarchy_device(int T, int L, DeviceHierarchy *out, std::string *err,
                           cudaStream_t stream) {
  if (T < 1 || T > kMaxTerms || L < 0 || L > kMaxTier) {
    *err = "hierarchy: terms must be in [1, 64] and tiers in [0, 250]";
    return 1;
  }
  const int amax = L + T + 1, width = T + 2;
  std::vector<unsigned long long> tab((size_t)(amax + 1) * width, 0ull);
  const unsigned long long kCap = 1ull << 62;
  for (int a = 0; a <= amax; ++a) {
    tab[(size_t)a * width] = 1;
    for (int b = 1; b < width && b <= a; ++b) {
      unsigned long long v = tab[(size_t)(a - 1) * width + b - 1] +
                             (b <= a - 1 ? tab[(size_t)(a - 1) * width + b] : 0ull);
      tab[(size_t)a * width + b] = v > kCap ? kCap : v;
    }
  }
  std::vector<long long> count(L + 1), first(L + 2);
  long long M = 0;
  for (int l = 0; l <= L; ++l) {
    unsigned long long c = tab[(size_t)(l + T - 1) * width + (T - 1)];
    if (c >= (1ull << 31)) {
      *err = "hierarchy: a tier exceeds 2^31 nodes";
      return 3;
    }
    count[l] = (long long)c;
    first[l] = M;
    M += count[l];
    if (M >= (1ll << 31)) {
      *err = "hierarchy: more than 2^31 nodes";
      return 3;
    }
  }
  first[L + 1] = M;
  out->M = M;
  out->T = T;
  out->L = L;
  out->tier_count = count;
  out->tier_first = first;
  if (out->budget > 0 && M > out->budget) {
    *err = "hierarchy: " + std::to_string(M) + " nodes exceed the node budget of " +
           std::to_string(out->budget);
    return 3;
  }

  DeviceBuffer d_tab, d_first_q, d_keep, d_bsum, d_total, d_tfirst, d_bad;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t x) { if (x != cudaSuccess && e == cudaSuccess) e = x; };
  // 64 bytes past the end of each table: the tiled kernels bulk-copy a
  // tile's records as a 16-byte aligned window, which may reach up to 15
  // bytes past the last record.
  chk(out->mi.alloc((size_t)M * T + 64));
  chk(out->next.alloc((size_t)M * T * sizeof(int32_t) + 64));
  chk(out->prev.alloc((size_t)M * T * sizeof(int32_t) + 64));
  chk(out->rank_to_id.alloc((size_t)M * sizeof(int32_t)));
  chk(d_tab.alloc(tab.size() * sizeof(unsigned long long)));
  chk(d_tfirst.alloc((size_t)(L + 2) * sizeof(long long)));
  long long max_cand = 1;
  for (int l = 1; l <= L; ++l) max_cand = std::max(max_cand, (long long)T * count[l - 1]);
  long long max_count = 1;
  for (int l = 0; l <= L; ++l) max_count = std::max(max_count, count[l]);
  chk(d_first_q.alloc((size_t)max_count * sizeof(unsigned long long)));
  chk(d_keep.alloc((size_t)max_cand));
  chk(d_bsum.alloc((size_t)((max_cand + kScanBlock - 1) / kScanBlock + 1) * sizeof(long long)));
  chk(d_total.alloc(sizeof(long long)));
  chk(d_bad.alloc(sizeof(int)));
  if (e != cudaSuccess) {
    *err = std::string("hierarchy: device allocation failed: ") + cudaGetErrorString(e);
    return 2;
  }
  chk(cudaMemcpyAsync(d_tab.ptr, tab.data(), tab.size() * sizeof(unsigned long long),
                      cudaMemcpyHostToDevice, stream));
  chk(cudaMemcpyAsync(d_tfirst.ptr, first.data(), (size_t)(L + 2) * sizeof(long long),
                      cudaMemcpyHostToDevice, stream));
  uint8_t *mi = (uint8_t *)out->mi.ptr;
  int32_t *r2i = (int32_t *)out->rank_to_id.ptr;
  chk(cudaMemsetAsync(mi, 0, (size_t)T, stream));  // tier 0: the zero index
  chk(cudaMemsetAsync(d_bad.ptr, 0, sizeof(int), stream));
  const int32_t zero = 0;
  chk(cudaMemcpyAsync(r2i, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, stream));
  chk(cudaStreamSynchronize(stream));
  Binom binom{(const unsigned long long *)d_tab.ptr, width};

  for (int l = 1; l <= L; ++l) {
    const long long C = count[l - 1];
    const long long ncand = (long long)T * C;
    const long long nblk = (ncand + kScanBlock - 1) / kScanBlock;
    init_first_q_kernel<<<blocks_for(count[l], 256), 256, 0, stream>>>(
        (unsigned long long *)d_first_q.ptr, count[l]);
    first_occurrence_kernel<<<blocks_for(ncand, 256), 256, 0, stream>>>(
        mi, T, first[l - 1], C, ncand, binom, (unsigned long long *)d_first_q.ptr);
    keep_flags_kernel<<<(unsigned)nblk, kScanBlock, 0, stream>>>(
        mi, T, first[l - 1], C, ncand, binom, (const unsigned long long *)d_first_q.ptr,
        (uint8_t *)d_keep.ptr, (long long *)d_bsum.ptr);
    scan_block_sums_kernel<<<1, 1024, 0, stream>>>((long long *)d_bsum.ptr, nblk,
                                                   (long long *)d_total.ptr);
    scatter_tier_kernel<<<(unsigned)nblk, kScanBlock, 0, stream>>>(
        mi, T, first[l - 1], C, ncand, first[l], count[l], binom, (const uint8_t *)d_keep.ptr,
        (const long long *)d_bsum.ptr, r2i + first[l], d_bad.as<int>());
    long long got = 0;
    chk(cudaMemcpyAsync(&got, d_total.ptr, sizeof(long long), cudaMemcpyDeviceToHost, stream));
    chk(cudaStreamSynchronize(stream));
    chk(cudaGetLastError());
    if (e != cudaSuccess) {
      *err = std::string("hierarchy: CUDA error: ") + cudaGetErrorString(e);
      return 7;
    }
    if (got != count[l]) {
      *err = "hierarchy: tier " + std::to_string(l) + " produced " + std::to_string(got) +
             " nodes, expected " + std::to_string(count[l]);
      return 7;
    }
  }
  link_kernel<<<blocks_for(M, 128), 128, 0, stream>>>(
      mi, T, L, M, binom, (const long long *)d_tfirst.ptr, r2i, (int32_t *)out->next.ptr,
      (int32_t *)out->prev.ptr, d_bad.as<int>());
  chk(cudaGetLastError());
  int bad = 0;
  chk(cudaMemcpyAsync(&bad, d_bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, stream));
  chk(cudaStreamSynchronize(stream));
  if (e != cudaSuccess) {
    *err = std::string("hierarchy: CUDA error: ") + cudaGetErrorString(e);
    return 7;
  }
  if (bad) {
    *err = "hierarchy: construction produced an index outside its tier";
    return 7;
  }
  return 0;
}

}  // namespace phi
