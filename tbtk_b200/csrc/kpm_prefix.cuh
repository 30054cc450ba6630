// FP64 head of a mixed-precision doubling run.
//
// The doubling identities mu_{2m} = 2<j_m|j_m> - mu_0 and
// mu_{2m-1} = 2<j_m|j_{m-1}> - mu_1 (the moments of the reference's
// recursion, Lib/src/Solver/ChebyshevExpander.cpp:150-190, taken from half
// as many steps) pick up the FP32 rounding of the recursion vectors through
// whole-vector dot products.  The rounding that matters is that of the first
// few dozen steps, while j_n still sits on the few rows around its source
// with entries of order one: with those steps in FP64 the largest relative
// LDOS error of the doubling path drops about fourfold (1.6e-6 -> 3.9e-7 on
// 1000-point windows of s = 12, M = 512-4096 square and honeycomb lattices).
//
// So one block per source computes j_0 .. j_q in FP64 on the rows they reach
// (the ball of radius q around the source in the matrix graph, which needs a
// structurally symmetric pattern), writes the moments of those steps, and the
// FP32 recursion starts from j_{q-1}, j_q rounded once.  The rows live in a
// per-block open-addressing table (row -> local index) in shared memory, the
// three FP64 vectors in global scratch (L2-resident); every probe loop is
// bounded by the table size.  When the ball outgrows the table the block
// stops at the last complete step and reports it.  The dot products are
// summed in 64-bit fixed point (2^-61 units), so the moments do not depend
// on the order in which rows entered the table.
#pragma once

#include "kpm_kernels.cuh"

#include <algorithm>
#include <vector>

namespace tbtkkpm {

constexpr uint32_t kPrefixSteps = 32;      // FP64 steps of a doubling run's head
constexpr uint32_t kPrefixRows = 6144;     // rows of one source's ball
constexpr uint32_t kPrefixSlots = 8192;    // hash slots (power of two, above the rows)
constexpr uint32_t kPrefixSlotBits = 13;
constexpr uint32_t kPrefixEmpty = 0xffffffffu;
constexpr uint32_t kPrefixMaxJobs = 512;   // sources of one launch
constexpr int kPrefixBlock = 256;
constexpr double kPrefixFix = 2305843009213693952.0;          // 2^61
constexpr double kPrefixUnit = 1.0 / 2305843009213693952.0;   // 2^-61
// shared memory of a block: key[slots] u32 | rows[rows] u32 | index[slots] u16
constexpr size_t kPrefixSmem = (size_t)kPrefixSlots * 4 + (size_t)kPrefixRows * 4 + (size_t)kPrefixSlots * 2;
// global scratch of a source: v[3][rows] (j_{n-1}, j_n, j_{n+1} in rotation)
constexpr size_t kPrefixScratch = 3 * (size_t)kPrefixRows * sizeof(double2);

struct PrefixJob {
  const uint32_t *slice_ptr;  // the source's matrix (SELL-32 of 2H/s)
  const uint32_t *scol;
  const double2 *sval;
  uint32_t site;        // source row (and the moments' target row)
  uint32_t steps;       // j_0 .. j_steps wanted
  uint32_t M;           // doubled moments written for n < M
  uint32_t ld;          // direct moments written for n < ld
  double2 *mu;          // doubled-moment row
  double2 *mu_direct;   // direct-moment row
  void *x_cur, *x_prev; // [rows][W] buffers that take j_q and j_{q-1}
  uint32_t W, col;      // row stride and column of the source
  uint32_t real;        // buffers hold real floats (else complex64)
  uint32_t pad;
};

// Result of one source: the last step computed (q) and the rows used.
struct PrefixResult {
  uint32_t q, count;
};

__device__ __forceinline__ uint32_t prefix_hash(uint32_t row) {
  return (row * 2654435761u) >> (32 - kPrefixSlotBits);
}

__device__ __forceinline__ int prefix_find(const uint32_t *key, const uint16_t *index, uint32_t row) {
  uint32_t h = prefix_hash(row);
  for (uint32_t p = 0; p < kPrefixSlots; p++) {
    const uint32_t k = key[h];
    if (k == row) return (int)index[h];
    if (k == kPrefixEmpty) return -1;
    h = (h + 1) & (kPrefixSlots - 1);
  }
  return -1;
}

// Adds `row` to the ball unless present.  A new row gets the next local
// index with zero values in all three vectors; past kPrefixRows (or with no
// free slot) *over is set instead.
__device__ __forceinline__ void prefix_insert(uint32_t *key, uint16_t *index, uint32_t *rows,
                                              double2 *v, uint32_t row, uint32_t *count,
                                              uint32_t *over) {
  uint32_t h = prefix_hash(row);
  for (uint32_t p = 0; p < kPrefixSlots; p++) {
    const uint32_t prev = atomicCAS(key + h, kPrefixEmpty, row);
    if (prev == row) return;
    if (prev == kPrefixEmpty) {
      const uint32_t i = atomicAdd(count, 1u);
      if (i < kPrefixRows) {
        index[h] = (uint16_t)i;
        rows[i] = row;
        const double2 z = make_double2(0.0, 0.0);
        v[i] = z;
        v[kPrefixRows + i] = z;
        v[2 * (size_t)kPrefixRows + i] = z;
      } else {
        *over = 1;
      }
      return;
    }
    h = (h + 1) & (kPrefixSlots - 1);
  }
  *over = 1;
}

__device__ __forceinline__ long long prefix_block_sum(long long x, long long *red) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = x;
  __syncthreads();
  long long t = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < kPrefixBlock / 32; i++) t += red[i];
  return t;  // valid in thread 0
}

// One block per source (kPrefixSmem bytes of dynamic shared memory).
// j_1 = (H/s) j_0 takes half of the stored 2H/s (exact), later steps
// j_{n+1} = (2H/s) j_n - j_{n-1}; every product and sum in FP64 (fma), rows
// in the matrix's entry order.  With q >= 2 steps done, the block writes
// j_q and j_{q-1} into its column of the two recursion buffers (zero
// elsewhere beforehand), rounded once to FP32.
static __global__ void __launch_bounds__(kPrefixBlock)
kpm_prefix(const PrefixJob *__restrict__ jobs, char *scratch, PrefixResult *res) {
  extern __shared__ __align__(16) unsigned char prefix_smem[];
  __shared__ uint32_t s_count, s_over;
  __shared__ long long red[kPrefixBlock / 32];
  const PrefixJob &J = jobs[blockIdx.x];
  uint32_t *key = reinterpret_cast<uint32_t *>(prefix_smem);
  uint32_t *rows = key + kPrefixSlots;
  uint16_t *index = reinterpret_cast<uint16_t *>(rows + kPrefixRows);
  double2 *v = reinterpret_cast<double2 *>(scratch + (size_t)blockIdx.x * kPrefixScratch);
  for (uint32_t i = threadIdx.x; i < kPrefixSlots; i += kPrefixBlock) key[i] = kPrefixEmpty;
  if (threadIdx.x == 0) {
    s_count = 0;
    s_over = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    prefix_insert(key, index, rows, v, J.site, &s_count, &s_over);
    v[0] = make_double2(1.0, 0.0);
    if (J.M > 0) J.mu[0] = make_double2(1.0, 0.0);
    if (J.ld > 0) J.mu_direct[0] = make_double2(1.0, 0.0);
  }
  __syncthreads();
  uint32_t f0 = 0, f1 = 1, q = 0;
  double2 mu1 = make_double2(0.0, 0.0);
  for (uint32_t n = 0; n < J.steps; n++) {
    // rows of the next ball: neighbours of the last step's new rows
    for (uint32_t i = f0 + threadIdx.x; i < f1; i += kPrefixBlock) {
      const uint32_t r = rows[i], s = r >> 5, l = r & 31;
      const uint32_t cb = __ldg(J.slice_ptr + s), ce = __ldg(J.slice_ptr + s + 1);
      for (uint32_t k = cb; k < ce; k++) {
        const uint32_t c = __ldg(J.scol + (uint64_t)k * 32 + l);
        if (c != kPad) prefix_insert(key, index, rows, v, c, &s_count, &s_over);
      }
    }
    __syncthreads();
    if (s_over) break;
    const uint32_t cnt = s_count;
    const double2 *x = v + (size_t)(n % 3) * kPrefixRows;
    const double2 *y = v + (size_t)((n + 2) % 3) * kPrefixRows;
    double2 *out = v + (size_t)((n + 1) % 3) * kPrefixRows;
    long long sa = 0, sb = 0;
    for (uint32_t i = threadIdx.x; i < cnt; i += kPrefixBlock) {
      const uint32_t r = rows[i], s = r >> 5, l = r & 31;
      const uint32_t cb = __ldg(J.slice_ptr + s), ce = __ldg(J.slice_ptr + s + 1);
      double ax = 0.0, ay = 0.0;
      for (uint32_t k = cb; k < ce; k++) {
        const uint64_t slot = (uint64_t)k * 32 + l;
        const uint32_t c = __ldg(J.scol + slot);
        if (c == kPad) continue;
        const int j = prefix_find(key, index, c);
        if (j < 0) continue;
        const double2 a = __ldg(J.sval + slot), b = x[j];
        ax = fma(a.x, b.x, fma(-a.y, b.y, ax));
        ay = fma(a.x, b.y, fma(a.y, b.x, ay));
      }
      if (n == 0) {
        ax *= 0.5;
        ay *= 0.5;
      } else {
        ax -= y[i].x;
        ay -= y[i].y;
      }
      out[i] = make_double2(ax, ay);
      const double2 b = x[i];
      sa += __double2ll_rn(fma(ax, ax, ay * ay) * kPrefixFix);
      sb += __double2ll_rn(fma(ax, b.x, ay * b.y) * kPrefixFix);
    }
    const long long ta = prefix_block_sum(sa, red);
    const long long tb = prefix_block_sum(sb, red);
    if (threadIdx.x == 0) {
      const uint32_t m = n + 1;
      const double2 d = out[0];  // the source row has local index 0
      if (m < J.ld) J.mu_direct[m] = d;
      if (m == 1) {
        mu1 = d;
        if (J.M > 1) J.mu[1] = d;
      }
      const double a = (double)ta * kPrefixUnit, b = (double)tb * kPrefixUnit;
      if (2 * m < J.M) J.mu[2 * m] = make_double2(2.0 * a - 1.0, -0.0);
      if (m >= 2 && 2 * m - 1 < J.M) J.mu[2 * m - 1] = make_double2(2.0 * b - mu1.x, -mu1.y);
    }
    q = n + 1;
    f0 = f1;
    f1 = cnt;
    __syncthreads();
  }
  const uint32_t count = min(s_count, kPrefixRows);
  if (threadIdx.x == 0) res[blockIdx.x] = {q, count};
  if (q < 2) return;
  const double2 *cur = v + (size_t)(q % 3) * kPrefixRows;
  const double2 *prev = v + (size_t)((q - 1) % 3) * kPrefixRows;
  for (uint32_t i = threadIdx.x; i < count; i += kPrefixBlock) {
    const uint64_t o = (uint64_t)rows[i] * J.W + J.col;
    const double2 c = cur[i], p = prev[i];
    if (J.real) {
      static_cast<float *>(J.x_cur)[o] = __double2float_rn(c.x);
      static_cast<float *>(J.x_prev)[o] = __double2float_rn(p.x);
    } else {
      static_cast<float2 *>(J.x_cur)[o] = make_float2(__double2float_rn(c.x), __double2float_rn(c.y));
      static_cast<float2 *>(J.x_prev)[o] = make_float2(__double2float_rn(p.x), __double2float_rn(p.y));
    }
  }
}

// Structural symmetry of a CSR pattern (every (r, c) has a (c, r)), which
// the ball of kpm_prefix relies on.  Rows longer than kPrefixRows count as a
// failure (their scan is not done and such a ball would not fit anyway).
static __global__ void k_pattern_check(uint32_t N, const uint32_t *__restrict__ rowptr,
                                       const uint32_t *__restrict__ col, unsigned *flag) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const uint32_t e0 = rowptr[r], e1 = rowptr[r + 1];
  if (e1 - e0 > kPrefixRows) {
    atomicOr(flag, 1u);
    return;
  }
  for (uint32_t e = e0; e < e1; e++) {
    const uint32_t c = col[e];
    if (c >= N) {
      atomicOr(flag, 1u);
      return;
    }
    const uint32_t f0 = rowptr[c], f1 = rowptr[c + 1];
    if (f1 - f0 > kPrefixRows) {
      atomicOr(flag, 1u);
      return;
    }
    bool found = false;
    for (uint32_t f = f0; f < f1 && !found; f++) found = col[f] == r;
    if (!found) {
      atomicOr(flag, 1u);
      return;
    }
  }
}

}  // namespace tbtkkpm

#include "kpm_host.h"

namespace tbtkkpm {

// Runs the FP64 head of `jobs` on stream st, kPrefixMaxJobs sources per
// launch (the scratch is reused); every source with q >= 2 leaves j_q and
// j_{q-1} in its buffers.  res[i] receives the steps source i reached and
// its rows.  Returns after the stream has passed the last launch.
static int run_fp64_head(cudaStream_t st, const std::vector<PrefixJob> &jobs, Workspace &ws,
                         std::vector<PrefixResult> &res) {
  const size_t nj = jobs.size();
  res.assign(nj, PrefixResult{0, 0});
  if (nj == 0) return 0;
  const size_t chunk = std::min<size_t>(nj, kPrefixMaxJobs);
  int rc;
  if ((rc = ws.head.reserve(kPrefixScratch * chunk)) ||
      (rc = ws.head_jobs.reserve(sizeof(PrefixJob) * nj)) ||
      (rc = ws.head_res.reserve(sizeof(PrefixResult) * nj)))
    return rc;
  cudaError_t e = cudaFuncSetAttribute(kpm_prefix, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kPrefixSmem);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ws.head_jobs.ptr, jobs.data(), sizeof(PrefixJob) * nj, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "fp64 head: jobs");
  uint64_t launches = 0;
  for (size_t j0 = 0; j0 < nj; j0 += chunk) {
    const unsigned n = (unsigned)std::min(chunk, nj - j0);
    kpm_prefix<<<n, kPrefixBlock, kPrefixSmem, st>>>(ws.head_jobs.as<PrefixJob>() + j0, ws.head.as<char>(),
                                                     ws.head_res.as<PrefixResult>() + j0);
    launches++;
  }
  count_launches(launches);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "fp64 head: launch");
  e = cudaMemcpyAsync(res.data(), ws.head_res.ptr, sizeof(PrefixResult) * nj, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "fp64 head");
  return 0;
}

}  // namespace tbtkkpm
