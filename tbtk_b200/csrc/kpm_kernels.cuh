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
// The VPT complex values a thread owns in one row of a batch, as raw loads:
// complex128 as double2 each; complex64 as float2 (VPT = 1) or float4 pairs.
// Ownership is interleaved: chunk q of thread `sub` of a TPR-thread group is
// chunk q*TPR + sub of the row, so every load instruction of the group reads
// one contiguous span (full 32-byte sectors) rather than strided pieces.
template <typename V, int TPR, int VPT> struct Pack;

template <int TPR, int VPT> struct Pack<double2, TPR, VPT> {
  using L = double2;
  static constexpr int NL = VPT;
  __device__ __forceinline__ static uint32_t col_of(int sub, int j) { return j * TPR + sub; }
  // value j of `sub` holding batch column c, or -1
  __device__ __forceinline__ static int slot_of(int sub, uint32_t c) {
    return (int)(c % TPR) == sub ? (int)(c / TPR) : -1;
  }
  __device__ __forceinline__ static void load(const double2 *row, int sub, L (&o)[NL]) {
#pragma unroll
    for (int j = 0; j < NL; j++) o[j] = __ldg(row + j * TPR + sub);
  }
  __device__ __forceinline__ static void load_rw(const double2 *row, int sub, L (&o)[NL]) {
#pragma unroll
    for (int j = 0; j < NL; j++) o[j] = row[j * TPR + sub];
  }
  __device__ __forceinline__ static double2 get(const L (&o)[NL], int j) { return o[j]; }
  // Stores v and returns the values as stored.
  __device__ __forceinline__ static void store(double2 *row, int sub, double2 (&v)[VPT]) {
#pragma unroll
    for (int j = 0; j < VPT; j++) row[j * TPR + sub] = v[j];
  }
};

template <int TPR, int VPT> struct Pack<float2, TPR, VPT> {
  static_assert(VPT == 1 || VPT % 2 == 0, "complex64 packs are 8 B or multiples of 16 B");
  using L = typename std::conditional<VPT == 1, float2, float4>::type;
  static constexpr int NL = VPT == 1 ? 1 : VPT / 2;
  __device__ __forceinline__ static uint32_t col_of(int sub, int j) {
    if constexpr (VPT == 1) return sub;
    else return (uint32_t)(((j >> 1) * TPR + sub) * 2 + (j & 1));
  }
  __device__ __forceinline__ static int slot_of(int sub, uint32_t c) {
    if constexpr (VPT == 1) {
      return (int)c == sub ? 0 : -1;
    } else {
      const uint32_t p = c >> 1;
      return (int)(p % TPR) == sub ? (int)(p / TPR) * 2 + (int)(c & 1) : -1;
    }
  }
  __device__ __forceinline__ static void load(const float2 *row, int sub, L (&o)[NL]) {
    const L *q = reinterpret_cast<const L *>(row);
#pragma unroll
    for (int j = 0; j < NL; j++) o[j] = __ldg(q + j * TPR + sub);
  }
  __device__ __forceinline__ static void load_rw(const float2 *row, int sub, L (&o)[NL]) {
    const L *q = reinterpret_cast<const L *>(row);
#pragma unroll
    for (int j = 0; j < NL; j++) o[j] = q[j * TPR + sub];
  }
  __device__ __forceinline__ static double2 get(const L (&o)[NL], int j) {
    if constexpr (VPT == 1) {
      return make_double2(o[0].x, o[0].y);
    } else {
      const float4 f = o[j >> 1];
      return (j & 1) ? make_double2(f.z, f.w) : make_double2(f.x, f.y);
    }
  }
  __device__ __forceinline__ static float2 getf(const L (&o)[NL], int j) {
    if constexpr (VPT == 1) {
      return o[0];
    } else {
      const float4 f = o[j >> 1];
      return (j & 1) ? make_float2(f.z, f.w) : make_float2(f.x, f.y);
    }
  }
  __device__ __forceinline__ static void storef(float2 *row, int sub, const float2 (&v)[VPT]) {
    if constexpr (VPT == 1) {
      row[sub] = v[0];
    } else {
      float4 *q = reinterpret_cast<float4 *>(row);
#pragma unroll
      for (int j = 0; j < VPT / 2; j++)
        q[j * TPR + sub] = make_float4(v[2 * j].x, v[2 * j].y, v[2 * j + 1].x, v[2 * j + 1].y);
    }
  }
  __device__ __forceinline__ static void store(float2 *row, int sub, double2 (&v)[VPT]) {
#pragma unroll
    for (int j = 0; j < VPT; j++)
      v[j] = make_double2((double)__double2float_rn(v[j].x), (double)__double2float_rn(v[j].y));
    if constexpr (VPT == 1) {
      row[sub] = make_float2((float)v[0].x, (float)v[0].y);
    } else {
      float4 *q = reinterpret_cast<float4 *>(row);
#pragma unroll
      for (int j = 0; j < VPT / 2; j++)
        q[j * TPR + sub] = make_float4((float)v[2 * j].x, (float)v[2 * j].y, (float)v[2 * j + 1].x,
                                       (float)v[2 * j + 1].y);
    }
  }
};

// Row entries a thread gathers at once.  With the register cap of one block
// per SM (MINB = 1) a whole tight-binding row (up to 8 entries) is in flight
// in one round trip; otherwise the count shrinks with the bytes per entry so
// the gathers fit the cap.
template <typename V, int VPT, int MINB> __host__ __device__ constexpr int entries_in_flight() {
  return MINB == 1 ? 8 : (sizeof(V) * VPT <= 16 ? 8 : (sizeof(V) * VPT <= 32 ? 4 : 2));
}

// ---------------------------------------------------------------- matrix / targets

struct Sell {
  const uint32_t *slice_ptr;  // [nslices + 1] chunk offsets (a chunk = 32 slots)
  const uint32_t *col;        // [chunks * 32], kPad in padding slots
  const double2 *val;         // [chunks * 32], 2H/s
  uint32_t N, nslices;
  const double *vre;          // [chunks * 32] real parts of val for a real matrix, else null
};

// ---------------------------------------------------------------- arithmetic
// How a step multiplies and accumulates.  Exact64: complex128 vectors, each
// operation rounded once in the reference's order.  Wide64: complex64
// vectors widened to FP64 in registers, FMA arithmetic, one rounding when
// the result is stored back to complex64.
struct Exact64 {
  using Acc = double2;
  using Val = double2;
  __device__ __forceinline__ static Val value(const Sell &A, uint64_t slot) {
    return __ldcs(A.val + slot);
  }
  __device__ __forceinline__ static Val half(Val v) { return make_double2(v.x * 0.5, v.y * 0.5); }
  __device__ __forceinline__ static Acc mac(Acc acc, Val v, Acc x) {
    return cadd_exact(acc, cmul_exact(v, x));
  }
  __device__ __forceinline__ static double2 wide(Acc a) { return a; }
};

struct Wide64 {
  using Acc = double2;
  using Val = double2;
  __device__ __forceinline__ static Val value(const Sell &A, uint64_t slot) {
    return __ldcs(A.val + slot);
  }
  __device__ __forceinline__ static Val half(Val v) { return make_double2(v.x * 0.5, v.y * 0.5); }
  __device__ __forceinline__ static Acc mac(Acc acc, Val v, Acc x) { return cmac<false>(acc, v, x); }
  __device__ __forceinline__ static double2 wide(Acc a) { return a; }
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
// The matrix holds 2H/s (the reference's stored values after `*= 2`); FIRST
// uses half of it, which is exact.  With Exact64 each element sees the
// reference's operations in the reference's order (acc = -y; acc += v*x
// for ascending columns), each rounded once, so the FP64 result is
// bit-identical to calculateCoefficientsCPU.
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
// conj(j_{n+1}) j_n per column, accumulated in FP64, to
// dots[blockIdx.x][2][Bp] (values as stored).

template <typename P, typename Acc, typename L, int NL>
__device__ __forceinline__ Acc pack_get(const L (&o)[NL], int j) {
  if constexpr (std::is_same<Acc, float2>::value) return P::getf(o, j);
  else return P::get(o, j);
}

// Stores the accumulators; afterwards acc holds the values as stored.
template <typename P, typename V, typename Acc, int VPT>
__device__ __forceinline__ void pack_store(V *row, int sub, Acc (&acc)[VPT]) {
  if constexpr (std::is_same<Acc, float2>::value) P::storef(row, sub, acc);
  else P::store(row, sub, acc);
}

// j_{n-1} is prefetched a row ahead when a thread's share of it is at most
// 64 bytes: measured faster than loading it at the start of its own row for
// every compiled shape, including (8, 8) complex64 where the second copy
// costs spills.
template <typename V, int VPT> __host__ __device__ constexpr bool prefetch_y() {
  return sizeof(V) * VPT <= 64;
}

// The prefetched part of a row: slice bounds, first entries and (see
// prefetch_y) j_{n-1}.
template <typename V, typename AR, int TPR, int VPT, int PF>
struct RowFetch {
  using L = typename Pack<V, TPR, VPT>::L;
  uint32_t row, l, cb, ce;
  bool ok, live;
  uint32_t cc[PF];  // column indices of entries sub + q*TPR (TPR > 1) or q (TPR == 1)
  typename AR::Val vv[TPR > 1 ? PF : 1];
  L yr[prefetch_y<V, VPT>() ? Pack<V, TPR, VPT>::NL : 1];
};

// Slice bounds of the row a thread takes in a tile.  They are loaded one
// tile before the row's entries, whose addresses depend on them, so the
// entry loads never wait for a bounds load.
struct RowBounds {
  uint32_t cb, ce;
};

template <int TPR>
__device__ __forceinline__ RowBounds load_bounds(const Sell &A, uint64_t tile, int grp) {
  constexpr int RPB = kBlock / TPR;
  const uint32_t s = (uint32_t)((tile * RPB + grp) >> 5);
  RowBounds b{0, 0};
  if (s < A.nslices) {
    b.cb = __ldg(A.slice_ptr + s);
    b.ce = __ldg(A.slice_ptr + s + 1);
  }
  return b;
}

template <typename V, typename AR, int TPR, int VPT, int PF, bool FIRST>
__device__ __forceinline__ void fetch_row(const Sell &A, uint32_t Bp, const V *y, uint64_t tile,
                                          int grp, int sub, RowBounds b,
                                          RowFetch<V, AR, TPR, VPT, PF> &f) {
  constexpr int RPB = kBlock / TPR;
  f.row = (uint32_t)(tile * RPB + grp);
  const uint32_t s = f.row >> 5;
  f.l = f.row & 31;
  f.ok = s < A.nslices;
  f.live = f.ok && f.row < A.N;
  f.cb = f.ce = 0;
  if (!f.ok) return;
  f.cb = b.cb;
  f.ce = b.ce;
#pragma unroll
  for (int q = 0; q < PF; q++) {
    const uint32_t k = TPR > 1 ? (uint32_t)(q * TPR + sub) : (uint32_t)q;
    f.cc[q] = (f.cb + k < f.ce) ? __ldcs(A.col + (uint64_t)(f.cb + k) * 32 + f.l) : kPad;
    if constexpr (TPR > 1)
      f.vv[q] = f.cc[q] != kPad ? AR::value(A, (uint64_t)(f.cb + k) * 32 + f.l)
                                : typename AR::Val{0, 0};
  }
  if constexpr (!FIRST && prefetch_y<V, VPT>())
    if (f.live) Pack<V, TPR, VPT>::load_rw(y + (uint64_t)f.row * Bp, sub, f.yr);
}

// j_{n-1} of the current row: the prefetched copy, or a load issued now.
template <typename V, typename AR, int TPR, int VPT, int PF>
__device__ __forceinline__ void row_y(const RowFetch<V, AR, TPR, VPT, PF> &f, const V *y,
                                      uint32_t Bp, int sub,
                                      typename Pack<V, TPR, VPT>::L (&out)[Pack<V, TPR, VPT>::NL]) {
  constexpr int NL = Pack<V, TPR, VPT>::NL;
  if constexpr (prefetch_y<V, VPT>()) {
#pragma unroll
    for (int q = 0; q < NL; q++) out[q] = f.yr[q];
  } else {
    if (f.live) Pack<V, TPR, VPT>::load_rw(y + (uint64_t)f.row * Bp, sub, out);
  }
}

template <typename V, typename AR, int TPR, int VPT, bool FIRST, bool DOTS, int MINB>
__global__ void __launch_bounds__(kBlock, MINB)
kpm_step(Sell A, uint32_t Bp, const V *__restrict__ x, V *__restrict__ y, Targets tg,
         uint32_t n_out, double2 *__restrict__ dots) {
  using P = Pack<V, TPR, VPT>;
  using L = typename P::L;
  using Acc = typename AR::Acc;
  using Val = typename AR::Val;
  constexpr int NL = P::NL;
  constexpr int G = entries_in_flight<V, VPT, MINB>();
  constexpr int RPB = kBlock / TPR;
  // entries per row prefetched: G for a thread-per-row, one per thread of
  // the group otherwise
  constexpr int PF = TPR == 1 ? G : 1;
  const int sub = threadIdx.x % TPR;
  const int grp = threadIdx.x / TPR;
  const unsigned mask = 0xffffffffu;
  // <j_{n+1}|j_{n+1}> and Re<j_{n+1}|j_n> per owned column (real for a
  // Hermitian H and a diagonal moment).  Kept in registers: measured 4-7%
  // faster for the (8, 8) complex64 shape than per-thread sums in shared
  // memory, although the registers cost about 200 spilled bytes there.
  double d_nn[DOTS ? VPT : 1], d_np[DOTS ? VPT : 1];
  if constexpr (DOTS) {
#pragma unroll
    for (int j = 0; j < VPT; j++) d_nn[j] = d_np[j] = 0.0;
  }
  // Slice bounds two tiles ahead (see load_bounds) for thread shares below
  // 64 bytes a row: measured 13% faster for complex128 B=1 and 4% for
  // complex64 (16, 4); the two registers cost the (8, 8) shape more spills
  // than the round trip they save, so it loads the bounds with the entries.
  constexpr bool PB = sizeof(V) * VPT < 64;
  const uint64_t ntiles = ((uint64_t)A.nslices * 32 + RPB - 1) / RPB;
  RowFetch<V, AR, TPR, VPT, PF> cur, nxt;
  RowBounds bn{0, 0};  // bounds of the next tile's row
  if (blockIdx.x < ntiles)
    fetch_row<V, AR, TPR, VPT, PF, FIRST>(A, Bp, y, blockIdx.x, grp, sub,
                                          load_bounds<TPR>(A, blockIdx.x, grp), cur);
  if constexpr (PB)
    if (blockIdx.x + gridDim.x < ntiles) bn = load_bounds<TPR>(A, blockIdx.x + gridDim.x, grp);
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    // issue the next row's loads (and the bounds of the one after) before
    // this row's gathers
    const uint64_t tnext = tile + gridDim.x, tnext2 = tnext + gridDim.x;
    RowBounds bn2{0, 0};
    if constexpr (PB) {
      if (tnext < ntiles) fetch_row<V, AR, TPR, VPT, PF, FIRST>(A, Bp, y, tnext, grp, sub, bn, nxt);
      if (tnext2 < ntiles) bn2 = load_bounds<TPR>(A, tnext2, grp);
    } else {
      if (tnext < ntiles)
        fetch_row<V, AR, TPR, VPT, PF, FIRST>(A, Bp, y, tnext, grp, sub,
                                              load_bounds<TPR>(A, tnext, grp), nxt);
    }
    // Whole warps past the last slice skip (the rows of a warp share a slice).
    if (cur.ok) {
      const uint32_t row = cur.row, l = cur.l, cb = cur.cb, ce = cur.ce, w = ce - cb;
      Acc acc[VPT];
      if constexpr (FIRST) {
#pragma unroll
        for (int j = 0; j < VPT; j++) acc[j] = Acc{0, 0};
      } else {
        L yv[NL];
        row_y(cur, y, Bp, sub, yv);
#pragma unroll
        for (int j = 0; j < VPT; j++) {
          const Acc v = cur.live ? pack_get<P, Acc>(yv, j) : Acc{0, 0};
          acc[j] = Acc{-v.x, -v.y};
        }
      }
      if constexpr (TPR == 1) {
        // entries [0, G) are prefetched; wider rows continue on demand
        for (uint32_t kb = 0; kb < w; kb += G) {
          uint32_t cc[G];
          Val vv[G];
          L raw[G][NL];
#pragma unroll
          for (int g = 0; g < G; g++)
            cc[g] = kb == 0 ? cur.cc[g]
                            : ((kb + g < w) ? __ldcs(A.col + (uint64_t)(cb + kb + g) * 32 + l) : kPad);
#pragma unroll
          for (int g = 0; g < G; g++)
            if (cc[g] != kPad) {
              vv[g] = AR::value(A, (uint64_t)(cb + kb + g) * 32 + l);
              P::load(x + (uint64_t)cc[g] * Bp, sub, raw[g]);
            }
#pragma unroll
          for (int g = 0; g < G; g++) {
            if (cc[g] == kPad) continue;
            Val v = vv[g];
            if constexpr (FIRST) v = AR::half(v);
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = AR::mac(acc[j], v, pack_get<P, Acc>(raw[g], j));
          }
        }
      } else {
        // entries [kb, kb + TPR): thread sub holds entry kb + sub
        for (uint32_t kb = 0; kb < w; kb += TPR) {
          uint32_t myc;
          Val myv;
          if (kb == 0) {
            myc = cur.cc[0];
            myv = cur.vv[0];
          } else {
            myc = kPad;
            myv = Val{0, 0};
            if (kb + sub < w) {
              myc = __ldcs(A.col + (uint64_t)(cb + kb + sub) * 32 + l);
              if (myc != kPad) myv = AR::value(A, (uint64_t)(cb + kb + sub) * 32 + l);
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
              if (cc[g] != kPad) P::load(x + (uint64_t)cc[g] * Bp, sub, raw[g]);
#pragma unroll
            for (int g = 0; g < G; g++) {
              const int src = (int)min(j0 + g, nk - 1);
              Val v;
              v.x = __shfl_sync(mask, myv.x, src, TPR);
              v.y = __shfl_sync(mask, myv.y, src, TPR);
              if (cc[g] == kPad) continue;
              if constexpr (FIRST) v = AR::half(v);
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[j] = AR::mac(acc[j], v, pack_get<P, Acc>(raw[g], j));
            }
          }
        }
      }
      if (cur.live) {
        // moments of flagged rows from the register values
        if (target_hit(tg, row)) {
          for (uint32_t i = target_first(tg, row); i < tg.count && __ldg(tg.row + i) == row; i++) {
            const int jt = P::slot_of(sub, __ldg(tg.col + i));
            if (jt >= 0) {
#pragma unroll
              for (int j = 0; j < VPT; j++)
                if (j == jt) tg.mu[(uint64_t)__ldg(tg.out + i) * tg.ld + n_out] = AR::wide(acc[j]);
            }
          }
        }
        if constexpr (DOTS && std::is_same<V, float2>::value) {
          // Round j_{n+1} to complex64 once, store it, and form both dot
          // products from the stored values: each term a complex64 product
          // summed in FP32 (one rounding of a 48-bit product per term, far
          // below the storage rounding the identities already carry) and
          // accumulated in FP64.  j_n of this row was just gathered by the
          // diagonal entry, so its reload hits L1.
          float2 af[VPT];
#pragma unroll
          for (int j = 0; j < VPT; j++)
            af[j] = make_float2(__double2float_rn(acc[j].x), __double2float_rn(acc[j].y));
          P::storef(y + (uint64_t)row * Bp, sub, af);
          L self[NL];
          P::load(x + (uint64_t)row * Bp, sub, self);
#pragma unroll
          for (int j = 0; j < VPT; j++) {
            const float2 b = P::getf(self, j);
            d_nn[j] += (double)fmaf(af[j].x, af[j].x, af[j].y * af[j].y);
            d_np[j] += (double)fmaf(af[j].x, b.x, af[j].y * b.y);
          }
        } else {
          pack_store<P, V, Acc, VPT>(y + (uint64_t)row * Bp, sub, acc);
          if constexpr (DOTS) {
            L self[NL];
            P::load(x + (uint64_t)row * Bp, sub, self);
#pragma unroll
            for (int j = 0; j < VPT; j++) {
              const double2 a = AR::wide(acc[j]), b = P::get(self, j);
              d_nn[j] = fma(a.x, a.x, fma(a.y, a.y, d_nn[j]));
              d_np[j] = fma(a.x, b.x, fma(a.y, b.y, d_np[j]));
            }
          }
        }
      }
    }
    cur = nxt;
    bn = bn2;
  }
  if constexpr (DOTS) {
    // Sum over the RPB groups of the block, one column at a time, in a fixed
    // order.
    __shared__ double red[kBlock][2];
#pragma unroll 1
    for (int j = 0; j < VPT; j++) {
      red[threadIdx.x][0] = d_nn[j];
      red[threadIdx.x][1] = d_np[j];
      __syncthreads();
      if (grp == 0) {
        double a = 0.0, b = 0.0;
        for (int r = 0; r < RPB; r++) {
          a += red[r * TPR + sub][0];
          b += red[r * TPR + sub][1];
        }
        double2 *o = dots + (uint64_t)blockIdx.x * 2 * Bp;
        const uint32_t c = P::col_of(sub, j);
        o[c] = make_double2(a, 0.0);
        o[Bp + c] = make_double2(b, 0.0);
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

// Real parts of the SELL values, and a flag set when some value has a
// nonzero imaginary part.
static __global__ void k_sell_real(uint64_t slots, const double2 *sval, double *sreal,
                                   unsigned *complex_flag) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= slots) return;
  const double2 v = sval[i];
  sreal[i] = v.x;
  if (v.y != 0.0) atomicOr(complex_flag, 1u);
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

// ---------------------------------------------------------------- table-free energy sums
// The sums of kpm_greens / kpm_ldos without the M x E table (an
// energy-sum variant for memory-light serving).  With x = E_e/s,
// theta = acos x, q = sin theta = sqrt(1 - x^2) and the table entries
// T[n][e] = (1/s)(-2i/q) e^{-i n theta}/(1 + delta_n0), every type is a
// combination of
//   C = sum_n c_n cos(n theta)/(1 + delta_n0) = sum_n a_n T_n(x)
//   S = sum_n c_n sin(n theta)/(1 + delta_n0) = q sum_{n>=1} c_n U_{n-1}(x),
// Retarded (-2/(s q))(S + iC), Advanced (-2/(s q))(S - iC), Principal
// (2/(s q)) S, NonPrincipal (2/(s q)) iC, LDOS Im(G_NP)/pi; S/q is formed
// without dividing by q.  C and S/q come from Clenshaw recurrences over
// descending n (b_n = a_n + 2x b_{n+1} - b_{n+2}; C = b_0 - x b_1 for the T
// series, b_0 for the U series), O(M) FMAs per (vector, energy) and no table
// traffic.  They differ from the table sums by rounding only (~1e-13
// relative at M = 4096).
template <int KT>
__global__ void __launch_bounds__(kEnergyBlock)
kpm_clenshaw(uint32_t M, uint32_t E, uint32_t K, const double *__restrict__ energies, double scale,
             const double2 *__restrict__ mu, int type, void *__restrict__ out) {
  __shared__ double2 cs[KT][kEnergyChunk];
  const uint32_t e = blockIdx.x * kEnergyBlock + threadIdx.x;
  const uint32_t k0 = blockIdx.y * KT;
  const double x = e < E ? energies[e] / scale : 0.0;
  const double x2 = 2.0 * x;
  double2 t1[KT], t2[KT], u1[KT], u2[KT];
#pragma unroll
  for (int j = 0; j < KT; j++) t1[j] = t2[j] = u1[j] = u2[j] = make_double2(0.0, 0.0);
  for (int64_t top = M; top > 0; top -= kEnergyChunk) {
    const uint32_t n0 = (uint32_t)(top > kEnergyChunk ? top - kEnergyChunk : 0);
    const uint32_t nc = (uint32_t)top - n0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < KT * kEnergyChunk; i += kEnergyBlock) {
      const uint32_t j = i / kEnergyChunk, n = i % kEnergyChunk;
      cs[j][n] = (k0 + j < K && n < nc) ? mu[(uint64_t)(k0 + j) * M + n0 + n] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (e < E) {
      for (int n = (int)nc - 1; n >= 0; n--) {
        const uint32_t nn = n0 + (uint32_t)n;
#pragma unroll
        for (int j = 0; j < KT; j++) {
          const double2 c = cs[j][n];
          if (nn >= 1) {
            const double2 bu = make_double2(fma(x2, u1[j].x, c.x - u2[j].x), fma(x2, u1[j].y, c.y - u2[j].y));
            u2[j] = u1[j];
            u1[j] = bu;
          }
          const double2 a = nn == 0 ? make_double2(0.5 * c.x, 0.5 * c.y) : c;
          const double2 bt = make_double2(fma(x2, t1[j].x, a.x - t2[j].x), fma(x2, t1[j].y, a.y - t2[j].y));
          t2[j] = t1[j];
          t1[j] = bt;
        }
      }
    }
  }
  if (e >= E) return;
  const double q = sqrt(1.0 - x * x);
  const double A = 2.0 / (scale * q), B = 2.0 / scale;  // C weight, S/q weight
#pragma unroll
  for (int j = 0; j < KT; j++) {
    if (k0 + j >= K) continue;
    const double2 C = make_double2(t1[j].x - x * t2[j].x, t1[j].y - x * t2[j].y);
    const double2 Sq = u1[j];  // S / q
    const uint64_t o = (uint64_t)(k0 + j) * E + e;
    if (type == 4) {
      static_cast<double *>(out)[o] = A * C.x / 3.14159265358979323846;
      continue;
    }
    double2 g;
    switch (type) {
      case 0:  // Advanced: -(2/(s q)) (S - iC)
        g = make_double2(-(B * Sq.x + A * C.y), -(B * Sq.y - A * C.x));
        break;
      case 1:  // Retarded: -(2/(s q)) (S + iC)
        g = make_double2(-(B * Sq.x - A * C.y), -(B * Sq.y + A * C.x));
        break;
      case 2:  // Principal: (2/(s q)) S
        g = make_double2(B * Sq.x, B * Sq.y);
        break;
      default:  // NonPrincipal: (2/(s q)) iC
        g = make_double2(-A * C.y, A * C.x);
    }
    static_cast<double2 *>(out)[o] = g;
  }
}

// ---------------------------------------------------------------- Chebyshev-node grid sums
// The sums of kpm_clenshaw on the grid of Chebyshev nodes x_k = cos(theta_k),
// theta_k = pi (2k + 1) / L, L = 2E (E a power of two), by one FFT per
// coefficient vector: O(L log L) arithmetic instead of O(M E).  With
// a_n = c_n / (1 + delta_n0),
//   F(k) = sum_n a_n e^{i n theta_k} = sum_{j<L} b_j e^{2 pi i j k / L},
//   b_j  = e^{i pi j / L} sum_{p} (-1)^p a_{j + p L}
// (e^{i pi (n + L) / L} = -e^{i pi n / L} folds M > L terms onto L), so one
// length-L DFT with a + exponent gives F(k) = sum a_n e^{+i n theta_k} at
// k < E and sum a_n e^{-i n theta_k} at L - 1 - k (theta_{L-1-k} = 2 pi -
// theta_k).  C = (F+ + F-)/2, S = (F+ - F-)/(2i), and the types combine as
// in kpm_clenshaw with A = 2/(s q) on both C and S.  Output energy e is node
// k = E - 1 - e, so the grid ascends: E_e = -s cos(pi (2e + 1) / L).
// tw[m] = e^{i pi m / L}, m < L (host libm).  One block per vector; the
// radix-2 decimation-in-time FFT runs in place in L complex doubles of
// dynamic shared memory (bit-reversed load, log2 L stages).
constexpr int kDctBlock = 512;
constexpr uint32_t kDctMaxE = 4096;  // L * 16 bytes = 128 KB of shared memory

static __global__ void __launch_bounds__(kDctBlock)
kpm_chebyshev_grid(uint32_t M, uint32_t E, uint32_t log2L, const double2 *__restrict__ tw,
                   double scale, const double2 *__restrict__ mu, int type, void *__restrict__ out) {
  extern __shared__ double2 fz[];
  const uint32_t L = 2 * E, vec = blockIdx.x;
  const double2 *c = mu + (uint64_t)vec * M;
  for (uint32_t j = threadIdx.x; j < L; j += kDctBlock) {
    double2 b = make_double2(0.0, 0.0);
    bool neg = false;
    for (uint32_t n = j; n < M; n += L, neg = !neg) {
      double2 a = __ldg(c + n);
      if (n == 0) a = make_double2(0.5 * a.x, 0.5 * a.y);
      b = neg ? make_double2(b.x - a.x, b.y - a.y) : make_double2(b.x + a.x, b.y + a.y);
    }
    const double2 w = __ldg(tw + j);
    const uint32_t r = log2L ? __brev(j) >> (32 - log2L) : 0;
    fz[r] = make_double2(b.x * w.x - b.y * w.y, b.x * w.y + b.y * w.x);
  }
  __syncthreads();
  for (uint32_t lh = 0; lh < log2L; lh++) {
    const uint32_t h = 1u << lh;
    for (uint32_t i = threadIdx.x; i < L / 2; i += kDctBlock) {
      const uint32_t r = i & (h - 1), i0 = ((i >> lh) << (lh + 1)) + r, i1 = i0 + h;
      const double2 w = __ldg(tw + (r << (log2L - lh)));  // e^{i pi r / h}
      const double2 u = fz[i0], v0 = fz[i1];
      const double2 v = make_double2(v0.x * w.x - v0.y * w.y, v0.x * w.y + v0.y * w.x);
      fz[i0] = make_double2(u.x + v.x, u.y + v.y);
      fz[i1] = make_double2(u.x - v.x, u.y - v.y);
    }
    __syncthreads();
  }
  for (uint32_t k = threadIdx.x; k < E; k += kDctBlock) {
    const double2 fp = fz[k], fm = fz[L - 1 - k];
    const double2 C = make_double2(0.5 * (fp.x + fm.x), 0.5 * (fp.y + fm.y));
    const double2 S = make_double2(0.5 * (fp.y - fm.y), -0.5 * (fp.x - fm.x));
    const double q = __ldg(&tw[2 * k + 1].y);  // sin(theta_k) > 0
    const double A = 2.0 / (scale * q);
    const uint64_t o = (uint64_t)vec * E + (E - 1 - k);
    if (type == 4) {
      static_cast<double *>(out)[o] = A * C.x / 3.14159265358979323846;
      continue;
    }
    double2 g;
    switch (type) {
      case 0:  // Advanced: -A (S - iC)
        g = make_double2(-A * (S.x + C.y), -A * (S.y - C.x));
        break;
      case 1:  // Retarded: -A (S + iC)
        g = make_double2(-A * (S.x - C.y), -A * (S.y + C.x));
        break;
      case 2:  // Principal: A S
        g = make_double2(A * S.x, A * S.y);
        break;
      default:  // NonPrincipal: A iC
        g = make_double2(-A * C.y, A * C.x);
    }
    static_cast<double2 *>(out)[o] = g;
  }
}

}  // namespace tbtkkpm
