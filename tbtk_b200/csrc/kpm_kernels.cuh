// Device kernels of the KPM (Chebyshev) path for sm_100a.
//
// The recursion is HBM-bandwidth bound (sparse SpMV/SpMM, ~0.1-1 flop/B), so
// the kernels are organised around bytes:
// * the Hamiltonian is stored as sliced ELL with 32-row slices (SELL-32):
//   entry k of row r lives at (slice_ptr[r/32] + k)*32 + r%32, so a warp that
//   owns a slice reads 128 B of column indices and 512 B of values per
//   instruction; it is read once per step and shared by the whole batch;
// * the vectors of a batch are interleaved [N][Bp], so a gathered row is one
//   contiguous, 16-byte aligned span;
// * all entries of a row (up to G at a time) are fetched before the gathers
//   are issued, so a thread keeps G independent loads in flight instead of a
//   col -> x dependency chain per entry;
// * j_{n+1} = 2H j_n - j_{n-1} overwrites j_{n-1} in place (two vector
//   buffers);
// * the moments <to|j_n> are taken from the FP64 register value of the row
//   that produces them, flagged by a bitmap, so no O(N) scan runs per step
//   (the reference scans a coefficient map of N ints every step,
//   Lib/src/cuda/ChebyshevSolver.cu:47-62);
// * for diagonal (LDOS) requests the kernel can also form the per-block
//   partial dot products <j_{n+1}|j_{n+1}> and <j_{n+1}|j_n> that give two
//   moments per step (mu_{2n+2} = 2<j_{n+1}|j_{n+1}> - mu_0,
//   mu_{2n+1} = 2<j_{n+1}|j_n> - mu_1), halving the steps.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tbtkkpm {

constexpr uint32_t kPad = 0xffffffffu;  // column index of a padding slot
constexpr int kBlock = 256;             // threads per recursion block

// ---------------------------------------------------------------- complex FP64
// Exact forms: one rounding per operation, no contraction, in the order
// GCC evaluates std::complex<double> (ac - bd, ad + bc).

__device__ __forceinline__ double2 cmul_exact(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

__device__ __forceinline__ double2 cadd_exact(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}

// acc += v*x, exactly as the reference (EXACT) or with FMA.
template <bool EXACT>
__device__ __forceinline__ double2 cmac(double2 acc, double2 v, double2 x) {
  if constexpr (EXACT) {
    return cadd_exact(acc, cmul_exact(v, x));
  } else {
    acc.x = fma(v.x, x.x, fma(-v.y, x.y, acc.x));
    acc.y = fma(v.x, x.y, fma(v.y, x.x, acc.y));
    return acc;
  }
}

// ---------------------------------------------------------------- vector packs
// VPT consecutive complex values of one row as raw loads: complex128 as
// double2 each; complex64 as float2 (VPT = 1) or float4 pairs.
template <typename V, int VPT> struct Pack;

template <int VPT> struct Pack<double2, VPT> {
  using L = double2;
  static constexpr int NL = VPT;
  __device__ __forceinline__ static void load(const double2 *p, L (&o)[NL]) {
#pragma unroll
    for (int j = 0; j < NL; j++) o[j] = __ldg(p + j);
  }
  __device__ __forceinline__ static void load_rw(const double2 *p, L (&o)[NL]) {
#pragma unroll
    for (int j = 0; j < NL; j++) o[j] = p[j];
  }
  __device__ __forceinline__ static double2 get(const L (&o)[NL], int j) { return o[j]; }
  // Stores v and returns the values as stored.
  __device__ __forceinline__ static void store(double2 *p, double2 (&v)[VPT]) {
#pragma unroll
    for (int j = 0; j < VPT; j++) p[j] = v[j];
  }
};

template <int VPT> struct Pack<float2, VPT> {
  static_assert(VPT == 1 || VPT % 2 == 0, "complex64 packs are 8 B or multiples of 16 B");
  using L = typename std::conditional<VPT == 1, float2, float4>::type;
  static constexpr int NL = VPT == 1 ? 1 : VPT / 2;
  __device__ __forceinline__ static void load(const float2 *p, L (&o)[NL]) {
    const L *q = reinterpret_cast<const L *>(p);
#pragma unroll
    for (int j = 0; j < NL; j++) o[j] = __ldg(q + j);
  }
  __device__ __forceinline__ static void load_rw(const float2 *p, L (&o)[NL]) {
    const L *q = reinterpret_cast<const L *>(p);
#pragma unroll
    for (int j = 0; j < NL; j++) o[j] = q[j];
  }
  __device__ __forceinline__ static double2 get(const L (&o)[NL], int j) {
    if constexpr (VPT == 1) {
      return make_double2(o[0].x, o[0].y);
    } else {
      const float4 f = o[j >> 1];
      return (j & 1) ? make_double2(f.z, f.w) : make_double2(f.x, f.y);
    }
  }
  __device__ __forceinline__ static void store(float2 *p, double2 (&v)[VPT]) {
#pragma unroll
    for (int j = 0; j < VPT; j++)
      v[j] = make_double2((double)__double2float_rn(v[j].x), (double)__double2float_rn(v[j].y));
    if constexpr (VPT == 1) {
      p[0] = make_float2((float)v[0].x, (float)v[0].y);
    } else {
      float4 *q = reinterpret_cast<float4 *>(p);
#pragma unroll
      for (int j = 0; j < VPT / 2; j++)
        q[j] = make_float4((float)v[2 * j].x, (float)v[2 * j].y, (float)v[2 * j + 1].x,
                           (float)v[2 * j + 1].y);
    }
  }
};

// Entries in flight per thread: about 16-32 B of vector data per entry.
template <typename V, int VPT> __host__ __device__ constexpr int entries_in_flight() {
  return sizeof(V) * VPT <= 16 ? 8 : (sizeof(V) * VPT <= 32 ? 4 : 2);
}

// ---------------------------------------------------------------- matrix / targets

struct Sell {
  const uint32_t *slice_ptr;  // [nslices + 1] chunk offsets (a chunk = 32 slots)
  const uint32_t *col;        // [chunks * 32], kPad in padding slots
  const double2 *val;         // [chunks * 32], 2H/s
  uint32_t N, nslices;
};

// Rows whose moments are wanted: bit r of `bitmap` is set when row r is the
// to-index of some request; row[] (sorted ascending), col[] (the batch
// column of the owning source) and out[] (output slot) list them.
struct Targets {
  const uint32_t *bitmap;
  const uint32_t *row;
  const uint32_t *col;
  const uint32_t *out;
  uint32_t count;
  double2 *mu;  // [K][ld] moments
  uint32_t ld;  // leading dimension of mu
};

__device__ __forceinline__ bool target_hit(const Targets &t, uint32_t r) {
  return (__ldg(t.bitmap + (r >> 5)) >> (r & 31)) & 1u;
}

__device__ __forceinline__ uint32_t target_first(const Targets &t, uint32_t r) {
  uint32_t lo = 0, hi = t.count;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(t.row + mid) < r) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------- recursion step
// One step of the three-term recursion for a batch of Bp = TPR*VPT vectors
// stored [N][Bp]:
//   FIRST: y = (H/s) x          (|j1> = H~|j0>, ChebyshevExpander.cpp:160)
//   else:  y = (2H/s) x - y     (:172-174; y holds j_{n-1} on entry)
// val holds 2H/s (the reference's stored values after `*= 2`); FIRST uses
// val * 0.5, which is exact.
// EXACT: per element the reference's operations in the reference's order
// (acc = -y; acc += v*x for ascending columns), each rounded once, so the
// FP64 result is bit-identical to calculateCoefficientsCPU.  Otherwise FMA.
//
// A group of TPR consecutive threads owns one row; thread `sub` of the group
// owns batch columns [sub*VPT, sub*VPT + VPT).  Blocks stride over tiles of
// kBlock/TPR rows.  While a row's gathers are in flight the thread has
// already issued the loads of its next row's column indices (and, for
// TPR > 1, values) and of its next j_{n-1} values, so each row costs one
// memory round trip instead of a column-index -> gather chain.
// MINB is the minimum number of resident blocks the compiler must allow
// (register cap), a tuning parameter.
// DOTS: each block writes its partial sums of conj(j_{n+1}) j_{n+1} and
// conj(j_{n+1}) j_n per column to dots[blockIdx.x][2][Bp] (values as stored).

// The prefetched part of a row: slice bounds, first entries, j_{n-1}.
template <typename V, int TPR, int VPT, int PF>
struct RowFetch {
  using L = typename Pack<V, VPT>::L;
  uint32_t row, l, cb, ce;
  bool ok, live;
  uint32_t cc[PF];      // column indices of entries sub + q*TPR (TPR > 1) or q (TPR == 1)
  double2 vv[TPR > 1 ? PF : 1];
  L yr[Pack<V, VPT>::NL];
};

template <typename V, int TPR, int VPT, int PF, bool FIRST>
__device__ __forceinline__ void fetch_row(const Sell &A, uint32_t Bp, const V *y, uint64_t tile,
                                          int grp, int sub, RowFetch<V, TPR, VPT, PF> &f) {
  constexpr int RPB = kBlock / TPR;
  f.row = (uint32_t)(tile * RPB + grp);
  const uint32_t s = f.row >> 5;
  f.l = f.row & 31;
  f.ok = s < A.nslices;
  f.live = f.ok && f.row < A.N;
  f.cb = f.ce = 0;
  if (!f.ok) return;
  f.cb = __ldg(A.slice_ptr + s);
  f.ce = __ldg(A.slice_ptr + s + 1);
#pragma unroll
  for (int q = 0; q < PF; q++) {
    const uint32_t k = TPR > 1 ? (uint32_t)(q * TPR + sub) : (uint32_t)q;
    f.cc[q] = (f.cb + k < f.ce) ? __ldcs(A.col + (uint64_t)(f.cb + k) * 32 + f.l) : kPad;
    if constexpr (TPR > 1)
      f.vv[q] = f.cc[q] != kPad ? __ldcs(A.val + (uint64_t)(f.cb + k) * 32 + f.l)
                                : make_double2(0.0, 0.0);
  }
  if constexpr (!FIRST)
    if (f.live) Pack<V, VPT>::load_rw(y + (uint64_t)f.row * Bp + sub * VPT, f.yr);
}

template <typename V, int TPR, int VPT, bool EXACT, bool FIRST, bool DOTS, int MINB>
__global__ void __launch_bounds__(kBlock, MINB)
kpm_step(Sell A, uint32_t Bp, const V *__restrict__ x, V *__restrict__ y, Targets tg,
         uint32_t n_out, double2 *__restrict__ dots) {
  using P = Pack<V, VPT>;
  using L = typename P::L;
  constexpr int NL = P::NL;
  constexpr int G = entries_in_flight<V, VPT>();
  constexpr int RPB = kBlock / TPR;
  // entries per row prefetched: G for a thread-per-row, one per thread of
  // the group otherwise
  constexpr int PF = TPR == 1 ? G : 1;
  const int sub = threadIdx.x % TPR;
  const int grp = threadIdx.x / TPR;
  const uint32_t c0 = sub * VPT;
  const unsigned mask = 0xffffffffu;
  double2 d_nn[DOTS ? VPT : 1], d_np[DOTS ? VPT : 1];
  if constexpr (DOTS) {
#pragma unroll
    for (int j = 0; j < VPT; j++) d_nn[j] = d_np[j] = make_double2(0.0, 0.0);
  }
  const uint64_t ntiles = ((uint64_t)A.nslices * 32 + RPB - 1) / RPB;
  RowFetch<V, TPR, VPT, PF> cur, nxt;
  if (blockIdx.x < ntiles) fetch_row<V, TPR, VPT, PF, FIRST>(A, Bp, y, blockIdx.x, grp, sub, cur);
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    // issue the next row's loads before this row's gathers
    const uint64_t tnext = tile + gridDim.x;
    if (tnext < ntiles) fetch_row<V, TPR, VPT, PF, FIRST>(A, Bp, y, tnext, grp, sub, nxt);
    // Whole warps past the last slice skip (the rows of a warp share a slice).
    if (cur.ok) {
      const uint32_t row = cur.row, l = cur.l, cb = cur.cb, ce = cur.ce, w = ce - cb;
      double2 acc[VPT];
#pragma unroll
      for (int j = 0; j < VPT; j++) {
        if constexpr (FIRST) {
          acc[j] = make_double2(0.0, 0.0);
        } else {
          const double2 v = cur.live ? P::get(cur.yr, j) : make_double2(0.0, 0.0);
          acc[j] = make_double2(-v.x, -v.y);
        }
      }
      L self[NL];
      bool have_self = false;
      if constexpr (TPR == 1) {
        // entries [0, G) are prefetched; wider rows continue on demand
        for (uint32_t kb = 0; kb < w; kb += G) {
          uint32_t cc[G];
          double2 vv[G];
          L raw[G][NL];
#pragma unroll
          for (int g = 0; g < G; g++)
            cc[g] = kb == 0 ? cur.cc[g]
                            : ((kb + g < w) ? __ldcs(A.col + (uint64_t)(cb + kb + g) * 32 + l) : kPad);
#pragma unroll
          for (int g = 0; g < G; g++)
            if (cc[g] != kPad) {
              vv[g] = __ldcs(A.val + (uint64_t)(cb + kb + g) * 32 + l);
              P::load(x + (uint64_t)cc[g] * Bp + c0, raw[g]);
            }
#pragma unroll
          for (int g = 0; g < G; g++) {
            if (cc[g] == kPad) continue;
            double2 v = vv[g];
            if constexpr (FIRST) v = make_double2(v.x * 0.5, v.y * 0.5);
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = cmac<EXACT>(acc[j], v, P::get(raw[g], j));
            if constexpr (DOTS) {
              if (cc[g] == row) {
#pragma unroll
                for (int q = 0; q < NL; q++) self[q] = raw[g][q];
                have_self = true;
              }
            }
          }
        }
      } else {
        // entries [kb, kb + TPR): thread sub holds entry kb + sub
        for (uint32_t kb = 0; kb < w; kb += TPR) {
          uint32_t myc;
          double2 myv;
          if (kb == 0) {
            myc = cur.cc[0];
            myv = cur.vv[0];
          } else {
            myc = kPad;
            myv = make_double2(0.0, 0.0);
            if (kb + sub < w) {
              myc = __ldcs(A.col + (uint64_t)(cb + kb + sub) * 32 + l);
              if (myc != kPad) myv = __ldcs(A.val + (uint64_t)(cb + kb + sub) * 32 + l);
            }
          }
          const uint32_t nk = min((uint32_t)TPR, w - kb);
          for (uint32_t j0 = 0; j0 < nk; j0 += G) {
            uint32_t cc[G];
            L raw[G][NL];
#pragma unroll
            for (int g = 0; g < G; g++) {
              cc[g] = __shfl_sync(mask, myc, (int)min(j0 + g, nk - 1), TPR);
              if (j0 + g >= nk) cc[g] = kPad;
            }
#pragma unroll
            for (int g = 0; g < G; g++)
              if (cc[g] != kPad) P::load(x + (uint64_t)cc[g] * Bp + c0, raw[g]);
#pragma unroll
            for (int g = 0; g < G; g++) {
              const int src = (int)min(j0 + g, nk - 1);
              double2 v;
              v.x = __shfl_sync(mask, myv.x, src, TPR);
              v.y = __shfl_sync(mask, myv.y, src, TPR);
              if (cc[g] == kPad) continue;
              if constexpr (FIRST) v = make_double2(v.x * 0.5, v.y * 0.5);
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[j] = cmac<EXACT>(acc[j], v, P::get(raw[g], j));
              if constexpr (DOTS) {
                if (cc[g] == row) {
#pragma unroll
                  for (int q = 0; q < NL; q++) self[q] = raw[g][q];
                  have_self = true;
                }
              }
            }
          }
        }
      }
      if (cur.live) {
        // moments of flagged rows from the FP64 register values
        if (target_hit(tg, row)) {
          for (uint32_t i = target_first(tg, row); i < tg.count && __ldg(tg.row + i) == row; i++) {
            const uint32_t bc = __ldg(tg.col + i);
            if (bc >= c0 && bc < c0 + VPT) {
#pragma unroll
              for (int j = 0; j < VPT; j++)
                if (bc == c0 + j) tg.mu[(uint64_t)__ldg(tg.out + i) * tg.ld + n_out] = acc[j];
            }
          }
        }
        P::store(y + (uint64_t)row * Bp + c0, acc);  // acc now holds the stored values
        if constexpr (DOTS) {
          if (!have_self) P::load(x + (uint64_t)row * Bp + c0, self);
#pragma unroll
          for (int j = 0; j < VPT; j++) {
            const double2 a = acc[j], b = P::get(self, j);
            d_nn[j].x = fma(a.x, a.x, fma(a.y, a.y, d_nn[j].x));
            d_np[j].x = fma(a.x, b.x, fma(a.y, b.y, d_np[j].x));
            d_np[j].y = fma(a.x, b.y, fma(-a.y, b.x, d_np[j].y));
          }
        }
      }
    }
    cur = nxt;
  }
  if constexpr (DOTS) {
    // Sum over the RPB groups of the block, one column at a time, in a fixed
    // order.
    __shared__ double2 red[kBlock][2];
#pragma unroll 1
    for (int j = 0; j < VPT; j++) {
      red[threadIdx.x][0] = d_nn[j];
      red[threadIdx.x][1] = d_np[j];
      __syncthreads();
      if (grp == 0) {
        double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
        for (int r = 0; r < RPB; r++) {
          const double2 u = red[r * TPR + sub][0], v = red[r * TPR + sub][1];
          a.x += u.x;
          b.x += v.x;
          b.y += v.y;
        }
        double2 *o = dots + (uint64_t)blockIdx.x * 2 * Bp;
        o[c0 + j] = a;
        o[Bp + c0 + j] = b;
      }
      __syncthreads();
    }
  }
}

// Two moments per step from the block partials of kpm_step<..., DOTS>:
// mu_{2m} = 2<j_m|j_m> - mu_0 and mu_{2m-1} = 2<j_m|j_{m-1}> - mu_1 for the
// step that produced j_m.  One block per batch column sums the partials in
// a fixed tree order (deterministic).  col_out[c] is the output slot of
// batch column c (or kPad).
constexpr int kFinalizeBlock = 128;
static __global__ void __launch_bounds__(kFinalizeBlock)
kpm_dots_finalize(uint32_t Bp, uint32_t nblocks, const double2 *__restrict__ dots,
                  const uint32_t *__restrict__ col_out, double2 *mu, uint32_t ld, uint32_t M,
                  uint32_t m) {
  const uint32_t c = blockIdx.x;
  const uint32_t slot = col_out[c];
  if (slot == kPad) return;
  __shared__ double ra[kFinalizeBlock], rbx[kFinalizeBlock], rby[kFinalizeBlock];
  double a = 0.0, bx = 0.0, by = 0.0;
  for (uint32_t k = threadIdx.x; k < nblocks; k += kFinalizeBlock) {
    a += dots[(uint64_t)k * 2 * Bp + c].x;
    const double2 v = dots[(uint64_t)k * 2 * Bp + Bp + c];
    bx += v.x;
    by += v.y;
  }
  ra[threadIdx.x] = a;
  rbx[threadIdx.x] = bx;
  rby[threadIdx.x] = by;
  __syncthreads();
  for (int h = kFinalizeBlock / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      ra[threadIdx.x] += ra[threadIdx.x + h];
      rbx[threadIdx.x] += rbx[threadIdx.x + h];
      rby[threadIdx.x] += rby[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double2 *row = mu + (uint64_t)slot * ld;
    const double2 mu0 = row[0], mu1 = row[1];
    if (2 * m < M) row[2 * m] = make_double2(2.0 * ra[0] - mu0.x, -mu0.y);
    if (m >= 2 && 2 * m - 1 < M)
      row[2 * m - 1] = make_double2(2.0 * rbx[0] - mu1.x, 2.0 * rby[0] - mu1.y);
  }
}

// Sets x[from_b][b] = 1 for each source (x zeroed beforehand) and the zeroth
// moments mu[k][0] = <to_k|from_owner> (ChebyshevExpander.cpp:153-157).
template <typename V>
__global__ void kpm_init_sources(uint32_t B, uint32_t Bp, const uint32_t *from, V *x,
                                 Targets tg) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B) {
    V one;
    one.x = 1;
    one.y = 0;
    x[(uint64_t)from[i] * Bp + i] = one;
  }
  if (i < tg.count) {
    const uint32_t b = tg.col[i];
    const double v = (tg.row[i] == from[b]) ? 1.0 : 0.0;
    tg.mu[(uint64_t)tg.out[i] * tg.ld] = make_double2(v, 0.0);
  }
}

// ---------------------------------------------------------------- SELL build
// Slice widths (longest row of each 32-row slice).
static __global__ void k_sell_width(uint32_t N, uint32_t nslices, const uint32_t *rowptr,
                             uint32_t *width) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslices) return;
  uint32_t w = 0;
  for (uint32_t r = s * 32; r < min(N, s * 32 + 32); r++) w = max(w, rowptr[r + 1] - rowptr[r]);
  width[s] = w;
}

// Scatter of the CSR rows into the slices; padding slots get kPad / 0.
static __global__ void k_sell_fill(uint32_t N, uint32_t nslices, const uint32_t *rowptr,
                            const uint32_t *col, const double2 *val, const uint32_t *slice_ptr,
                            uint32_t *scol, double2 *sval) {
  const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= (uint64_t)nslices * 32) return;
  const uint32_t s = (uint32_t)(r >> 5), l = (uint32_t)(r & 31);
  const uint32_t cb = slice_ptr[s], w = slice_ptr[s + 1] - cb;
  const uint32_t k0 = r < N ? rowptr[r] : 0, len = r < N ? rowptr[r + 1] - k0 : 0;
  for (uint32_t k = 0; k < w; k++) {
    const uint64_t slot = (uint64_t)(cb + k) * 32 + l;
    if (k < len) {
      scol[slot] = col[k0 + k];
      sval[slot] = val[k0 + k];
    } else {
      scol[slot] = kPad;
      sval[slot] = make_double2(0.0, 0.0);
    }
  }
}

// ---------------------------------------------------------------- damping
// mu[k][n] = mu[k][n]*a[n]/b component-wise (ChebyshevExpander.cpp:190-196);
// a[n] = sinh(lambda(1-n/M)) and b = sinh(lambda) come from the host's libm.
static __global__ void kpm_damp(uint32_t K, uint32_t M, const double *a, double b, double2 *mu) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint64_t)K * M) return;
  const uint32_t n = (uint32_t)(i % M);
  double2 c = mu[i];
  const double an = a[n];
  mu[i] = make_double2(__ddiv_rn(__dmul_rn(c.x, an), b), __ddiv_rn(__dmul_rn(c.y, an), b));
}

// ---------------------------------------------------------------- lookup table
// T[n][e] = (1/s)(-2i/sqrt(1-x^2)) exp(-i n acos x)/(1+delta_n0), x = E_e/s,
// with std::complex's evaluation order (ChebyshevExpander.cpp:258-268);
// acos and sincos are CUDA's, everything else is correctly rounded.
static __global__ void kpm_table_gen(uint32_t M, uint32_t E, const double *energies, double scale,
                                     double2 *table) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint64_t)M * E) return;
  const uint32_t n = (uint32_t)(i / E), e = (uint32_t)(i % E);
  const double x = __ddiv_rn(energies[e], scale);
  const double q = __dsqrt_rn(__dsub_rn(1.0, __dmul_rn(x, x)));
  const double is = __ddiv_rn(1.0, scale);
  // (1/s) * ((-2.*i) / q): (-0, -2)/q then scaled
  const double2 b = make_double2(__dmul_rn(is, __ddiv_rn(-0.0, q)), __dmul_rn(is, __ddiv_rn(-2.0, q)));
  const double th = acos(x);
  // -i * n * th: imaginary part (-n)*th, real part -0
  const double ang = __dmul_rn(-(double)n, th);
  double sn, cs;
  sincos(ang, &sn, &cs);
  double2 r = cmul_exact(b, make_double2(cs, sn));
  const double den = n == 0 ? 2.0 : 1.0;
  table[i] = make_double2(__ddiv_rn(r.x, den), __ddiv_rn(r.y, den));
}

// ---------------------------------------------------------------- energy sums
// G[k][e] accumulated over n ascending per (k, e), the reference's order
// (n outer, e inner, ChebyshevExpander.cpp:324-361), each operation rounded
// once.  KT coefficient vectors per thread share each table load; a block
// stages a chunk of their coefficients in shared memory.
constexpr int kEnergyBlock = 128;
constexpr int kEnergyChunk = 128;

template <int TYPE, int KT>
__global__ void __launch_bounds__(kEnergyBlock)
kpm_greens(uint32_t M, uint32_t E, uint32_t K, const double2 *__restrict__ table,
           const double2 *__restrict__ mu, double2 *__restrict__ G) {
  __shared__ double2 cs[KT][kEnergyChunk];
  const uint32_t e = blockIdx.x * kEnergyBlock + threadIdx.x;
  const uint32_t k0 = blockIdx.y * KT;
  double2 acc[KT];
#pragma unroll
  for (int j = 0; j < KT; j++) acc[j] = make_double2(0.0, 0.0);
  for (uint32_t n0 = 0; n0 < M; n0 += kEnergyChunk) {
    const uint32_t nc = min((uint32_t)kEnergyChunk, M - n0);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < KT * kEnergyChunk; i += kEnergyBlock) {
      const uint32_t j = i / kEnergyChunk, n = i % kEnergyChunk;
      double2 c = make_double2(0.0, 0.0);
      if (k0 + j < K && n < nc) c = mu[(uint64_t)(k0 + j) * M + n0 + n];
      if constexpr (TYPE == 3) {
        // c*i = (c.re*0 - c.im*1, c.re*1 + c.im*0)
        c = cmul_exact(c, make_double2(0.0, 1.0));
      }
      cs[j][n] = c;
    }
    __syncthreads();
    if (e < E) {
      for (uint32_t n = 0; n < nc; n++) {
        const double2 t = __ldg(table + (uint64_t)(n0 + n) * E + e);
#pragma unroll
        for (int j = 0; j < KT; j++) {
          const double2 c = cs[j][n];
          if constexpr (TYPE == 1) {          // Retarded: G += T*c
            acc[j] = cadd_exact(acc[j], cmul_exact(t, c));
          } else if constexpr (TYPE == 0) {   // Advanced: G += c*conj(T)
            acc[j] = cadd_exact(acc[j], cmul_exact(c, make_double2(t.x, -t.y)));
          } else if constexpr (TYPE == 2) {   // Principal: G += -c*Re(T)
            acc[j] = cadd_exact(acc[j], make_double2(__dmul_rn(-c.x, t.x), __dmul_rn(-c.y, t.x)));
          } else {                            // NonPrincipal: G -= (c*i)*Im(T)
            acc[j] = make_double2(__dsub_rn(acc[j].x, __dmul_rn(c.x, t.y)),
                                  __dsub_rn(acc[j].y, __dmul_rn(c.y, t.y)));
          }
        }
      }
    }
  }
  if (e < E) {
#pragma unroll
    for (int j = 0; j < KT; j++)
      if (k0 + j < K) G[(uint64_t)(k0 + j) * E + e] = acc[j];
  }
}

// LDOS[k][e] = 0 + Im(G_NP[k][e])/pi (PropertyExtractor ChebyshevExpander.cpp:682-683).
// Only the imaginary part of G_NonPrincipal is accumulated:
// Im(G) -= (c.re*1 + c.im*0) * Im(T).
template <int KT>
__global__ void __launch_bounds__(kEnergyBlock)
kpm_ldos(uint32_t M, uint32_t E, uint32_t K, const double2 *__restrict__ table,
         const double2 *__restrict__ mu, double *__restrict__ out) {
  __shared__ double cs[KT][kEnergyChunk];
  const uint32_t e = blockIdx.x * kEnergyBlock + threadIdx.x;
  const uint32_t k0 = blockIdx.y * KT;
  double acc[KT];
#pragma unroll
  for (int j = 0; j < KT; j++) acc[j] = 0.0;
  for (uint32_t n0 = 0; n0 < M; n0 += kEnergyChunk) {
    const uint32_t nc = min((uint32_t)kEnergyChunk, M - n0);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < KT * kEnergyChunk; i += kEnergyBlock) {
      const uint32_t j = i / kEnergyChunk, n = i % kEnergyChunk;
      double c = 0.0;
      if (k0 + j < K && n < nc) {
        const double2 m = mu[(uint64_t)(k0 + j) * M + n0 + n];
        c = __dadd_rn(__dmul_rn(m.x, 1.0), __dmul_rn(m.y, 0.0));
      }
      cs[j][n] = c;
    }
    __syncthreads();
    if (e < E) {
      for (uint32_t n = 0; n < nc; n++) {
        const double ti = __ldg(&table[(uint64_t)(n0 + n) * E + e].y);
#pragma unroll
        for (int j = 0; j < KT; j++) acc[j] = __dsub_rn(acc[j], __dmul_rn(cs[j][n], ti));
      }
    }
  }
  if (e < E) {
#pragma unroll
    for (int j = 0; j < KT; j++)
      if (k0 + j < K)
        out[(uint64_t)(k0 + j) * E + e] = __dadd_rn(0.0, __ddiv_rn(acc[j], 3.14159265358979323846));
  }
}

}  // namespace tbtkkpm
