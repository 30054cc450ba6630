// Device kernels of the KPM (Chebyshev) path for sm_100a.
//
// The recursion is HBM-bandwidth bound (sparse SpMV/SpMM, ~0.1-1 flop/B), so
// the kernels are organised around bytes: the Hamiltonian is read once per
// step and shared by every source vector of a batch; the vectors of a batch
// are interleaved [N][B] so a gathered row is one contiguous, 16-byte
// aligned span; the update j_{n+1} = 2H j_n - j_{n-1} overwrites j_{n-1} in
// place (two vector buffers, no third); the moments <to|j_n> are taken from
// the FP64 register value of the row that produces them, flagged by a bitmap
// (1 bit per row), so no O(N) scan runs per step (the reference scans a
// coefficient map of N ints every step, Lib/src/cuda/ChebyshevSolver.cu:47-62).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tbtkkpm {

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

// ---------------------------------------------------------------- storage
// Vector element types: complex128 (double2) or complex64 (float2).

template <typename V> struct VecTraits;
template <> struct VecTraits<double2> {
  __device__ __forceinline__ static double2 load(const double2 *p) { return __ldg(p); }
  __device__ __forceinline__ static double2 load_rw(const double2 *p) { return *p; }
  __device__ __forceinline__ static void store(double2 *p, double2 v) { *p = v; }
};
template <> struct VecTraits<float2> {
  __device__ __forceinline__ static double2 load(const float2 *p) {
    float2 f = __ldg(p);
    return make_double2(f.x, f.y);
  }
  __device__ __forceinline__ static double2 load_rw(const float2 *p) {
    float2 f = *p;
    return make_double2(f.x, f.y);
  }
  __device__ __forceinline__ static void store(float2 *p, double2 v) {
    *p = make_float2(__double2float_rn(v.x), __double2float_rn(v.y));
  }
};

// Loads VPT consecutive complex values of one row (VPT*sizeof(V) bytes,
// aligned to that size by construction of the [N][Bp] layout).
template <typename V, int VPT> struct RowChunk;
template <int VPT> struct RowChunk<double2, VPT> {
  __device__ __forceinline__ static void load(const double2 *p, double2 (&o)[VPT]) {
#pragma unroll
    for (int j = 0; j < VPT; j++) o[j] = __ldg(p + j);
  }
  __device__ __forceinline__ static void load_rw(const double2 *p, double2 (&o)[VPT]) {
#pragma unroll
    for (int j = 0; j < VPT; j++) o[j] = p[j];
  }
  __device__ __forceinline__ static void store(double2 *p, const double2 (&v)[VPT]) {
#pragma unroll
    for (int j = 0; j < VPT; j++) p[j] = v[j];
  }
};
template <int VPT> struct RowChunk<float2, VPT> {
  static_assert(VPT == 1 || VPT % 2 == 0, "complex64 chunks are 8 B or multiples of 16 B");
  __device__ __forceinline__ static void load(const float2 *p, double2 (&o)[VPT]) {
    if constexpr (VPT == 1) {
      float2 f = __ldg(p);
      o[0] = make_double2(f.x, f.y);
    } else {
      const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
      for (int j = 0; j < VPT / 2; j++) {
        float4 f = __ldg(q + j);
        o[2 * j] = make_double2(f.x, f.y);
        o[2 * j + 1] = make_double2(f.z, f.w);
      }
    }
  }
  __device__ __forceinline__ static void load_rw(const float2 *p, double2 (&o)[VPT]) {
    if constexpr (VPT == 1) {
      float2 f = *p;
      o[0] = make_double2(f.x, f.y);
    } else {
      const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
      for (int j = 0; j < VPT / 2; j++) {
        float4 f = q[j];
        o[2 * j] = make_double2(f.x, f.y);
        o[2 * j + 1] = make_double2(f.z, f.w);
      }
    }
  }
  __device__ __forceinline__ static void store(float2 *p, const double2 (&v)[VPT]) {
    if constexpr (VPT == 1) {
      p[0] = make_float2(__double2float_rn(v[0].x), __double2float_rn(v[0].y));
    } else {
      float4 *q = reinterpret_cast<float4 *>(p);
#pragma unroll
      for (int j = 0; j < VPT / 2; j++)
        q[j] = make_float4(__double2float_rn(v[2 * j].x), __double2float_rn(v[2 * j].y),
                           __double2float_rn(v[2 * j + 1].x), __double2float_rn(v[2 * j + 1].y));
    }
  }
};

// ---------------------------------------------------------------- targets
// Rows whose moments are wanted.  bitmap bit r is set when row r is the
// to-index of some request; tgt_row[] (sorted ascending) with tgt_col[]
// (the batch column = owning source) and tgt_out[] (output slot) list them.

struct Targets {
  const uint32_t *bitmap;   // ceil(N/32) words
  const uint32_t *row;      // [T] sorted
  const uint32_t *col;      // [T] batch column of the owning source
  const uint32_t *out;      // [T] output slot (to-index number)
  uint32_t count;
  double2 *mu;              // [K][M] moments
  uint32_t M;               // moments per to-index
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
// val2 holds 2H/s (the reference's stored values after `*= 2`); FIRST uses
// val2 * 0.5, which is exact.
// EXACT: per element the reference's operations in the reference's order
// (acc = -y; acc += v*x for ascending columns), each rounded once, so the
// FP64 result is bit-identical to calculateCoefficientsCPU.  Otherwise FMA.
// A group of TPR consecutive threads owns one row; thread `sub` of the group
// owns batch columns [sub*VPT, sub*VPT + VPT).
template <typename V, int TPR, int VPT, bool EXACT, bool FIRST>
__global__ void __launch_bounds__(256)
kpm_step(uint32_t N, uint32_t Bp, const uint32_t *__restrict__ rowptr,
         const uint32_t *__restrict__ col, const double2 *__restrict__ val2,
         const V *__restrict__ x, V *__restrict__ y, Targets tg, uint32_t n_out) {
  const uint64_t gt = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t row = (uint32_t)(gt / TPR);
  const uint32_t sub = (uint32_t)(gt % TPR);
  if (row >= N) return;
  const uint32_t c0 = sub * VPT;
  double2 acc[VPT];
  if constexpr (FIRST) {
#pragma unroll
    for (int j = 0; j < VPT; j++) acc[j] = make_double2(0.0, 0.0);
  } else {
    RowChunk<V, VPT>::load_rw(y + (uint64_t)row * Bp + c0, acc);
#pragma unroll
    for (int j = 0; j < VPT; j++) acc[j] = make_double2(-acc[j].x, -acc[j].y);
  }
  const uint32_t k0 = __ldg(rowptr + row), k1 = __ldg(rowptr + row + 1);
  for (uint32_t k = k0; k < k1; k++) {
    const uint32_t c = __ldcs(col + k);
    double2 v = __ldcs(val2 + k);
    if constexpr (FIRST) v = make_double2(v.x * 0.5, v.y * 0.5);
    double2 xv[VPT];
    RowChunk<V, VPT>::load(x + (uint64_t)c * Bp + c0, xv);
#pragma unroll
    for (int j = 0; j < VPT; j++) {
      if constexpr (EXACT) {
        acc[j] = cadd_exact(acc[j], cmul_exact(v, xv[j]));
      } else {
        acc[j].x = fma(v.x, xv[j].x, fma(-v.y, xv[j].y, acc[j].x));
        acc[j].y = fma(v.x, xv[j].y, fma(v.y, xv[j].x, acc[j].y));
      }
    }
  }
  RowChunk<V, VPT>::store(y + (uint64_t)row * Bp + c0, acc);
  if (target_hit(tg, row)) {
    for (uint32_t i = target_first(tg, row); i < tg.count && __ldg(tg.row + i) == row; i++) {
      const uint32_t bc = __ldg(tg.col + i);
      if (bc >= c0 && bc < c0 + VPT) {
#pragma unroll
        for (int j = 0; j < VPT; j++)
          if (bc == c0 + j) tg.mu[(uint64_t)__ldg(tg.out + i) * tg.M + n_out] = acc[j];
      }
    }
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
    one.x = 1; one.y = 0;
    x[(uint64_t)from[i] * Bp + i] = one;
  }
  if (i < tg.count) {
    const uint32_t b = tg.col[i];
    const double v = (tg.row[i] == from[b]) ? 1.0 : 0.0;
    tg.mu[(uint64_t)tg.out[i] * tg.M] = make_double2(v, 0.0);
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
// stages NC coefficients of its KT vectors in shared memory.
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
