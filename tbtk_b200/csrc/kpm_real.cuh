// Recursion step for real Hamiltonians at mixed precision: real float
// vectors, FP64 arithmetic.
//
// When every stored value 2H/s has a zero imaginary part and the sources are
// unit vectors (LDOS sites, moments from basis vectors), every Chebyshev
// vector j_n is real.  The complex64 step then only ever adds exact zeros to
// the imaginary parts, and its real parts are formed by the same FP64 FMAs
// in the same entry order as here, so this kernel returns the same values
// (moments, stored vectors, dot-product terms) as kpm_step<float2, Wide64>
// with half the vector bytes, half the FP32->FP64 conversions and a quarter
// of the FMAs.  Moments are written as complex (value, 0).
#pragma once

#include "kpm_kernels.cuh"

namespace tbtkkpm {

// The VPT real values a thread owns in a row of a batch: chunks of CS floats
// (CS = min(VPT, 4), loaded as float / float2 / float4), chunk q of thread
// `sub` being chunk q*TPR + sub of the row (interleaved, as Pack).
template <int TPR, int VPT> struct RPack {
  static constexpr int CS = VPT < 4 ? VPT : 4;
  static constexpr int NL = VPT / CS;
  using L = typename std::conditional<
      CS == 1, float, typename std::conditional<CS == 2, float2, float4>::type>::type;
  __device__ __forceinline__ static uint32_t col_of(int sub, int j) {
    return (uint32_t)(((j / CS) * TPR + sub) * CS + j % CS);
  }
  __device__ __forceinline__ static int slot_of(int sub, uint32_t c) {
    const uint32_t p = c / CS;
    return (int)(p % TPR) == sub ? (int)(p / TPR) * CS + (int)(c % CS) : -1;
  }
  __device__ __forceinline__ static void load(const float *row, int sub, L (&o)[NL]) {
    const L *q = reinterpret_cast<const L *>(row);
#pragma unroll
    for (int j = 0; j < NL; j++) o[j] = __ldg(q + j * TPR + sub);
  }
  __device__ __forceinline__ static void load_rw(const float *row, int sub, L (&o)[NL]) {
    const L *q = reinterpret_cast<const L *>(row);
#pragma unroll
    for (int j = 0; j < NL; j++) o[j] = q[j * TPR + sub];
  }
  __device__ __forceinline__ static float getf(const L (&o)[NL], int j) {
    if constexpr (CS == 1) {
      return o[j];
    } else if constexpr (CS == 2) {
      const float2 f = o[j >> 1];
      return (j & 1) ? f.y : f.x;
    } else {
      const float4 f = o[j >> 2];
      const int e = j & 3;
      return e == 0 ? f.x : (e == 1 ? f.y : (e == 2 ? f.z : f.w));
    }
  }
  __device__ __forceinline__ static void storef(float *row, int sub, const float (&v)[VPT]) {
    L *q = reinterpret_cast<L *>(row);
#pragma unroll
    for (int j = 0; j < NL; j++) {
      if constexpr (CS == 1) q[j * TPR + sub] = v[j];
      else if constexpr (CS == 2) q[j * TPR + sub] = make_float2(v[2 * j], v[2 * j + 1]);
      else
        q[j * TPR + sub] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
  }
};

template <int TPR, int VPT, int PF> struct RRowFetch {
  using L = typename RPack<TPR, VPT>::L;
  uint32_t row, l, cb, ce;
  bool ok, live;
  uint32_t cc[PF];
  double vv[TPR > 1 ? PF : 1];
  L yr[RPack<TPR, VPT>::NL];
};

template <int TPR, int VPT, int PF, bool FIRST, bool PFY = true>
__device__ __forceinline__ void rfetch_row(const Sell &A, uint32_t Bp, const float *y,
                                           uint64_t tile, int grp, int sub, RowBounds b,
                                           RRowFetch<TPR, VPT, PF> &f) {
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
      f.vv[q] = f.cc[q] != kPad ? __ldcs(A.vre + (uint64_t)(f.cb + k) * 32 + f.l) : 0.0;
  }
  if constexpr (!FIRST && PFY)
    if (f.live) RPack<TPR, VPT>::load_rw(y + (uint64_t)f.row * Bp, sub, f.yr);
}

// GIN: entries gathered per round trip (0: entries_in_flight's choice).
// OPT bit 0: load the slice bounds with the entries (not a tile ahead);
// bit 1: load j_{n-1} at the start of its row (not a row ahead); bit 3:
// the dot-product sums in this thread's slots of dynamic shared memory
// (2*VPT doubles per thread) instead of registers.
template <int TPR, int VPT, bool FIRST, bool DOTS, int MINB, int GIN = 0, int OPT = 0>
__global__ void __launch_bounds__(kBlock, MINB)
kpm_step_real(Sell A, uint32_t Bp, const float *__restrict__ x, float *__restrict__ y,
              Targets tg, uint32_t n_out, double2 *__restrict__ dots) {
  using P = RPack<TPR, VPT>;
  using L = typename P::L;
  constexpr int NL = P::NL;
  constexpr int G = GIN ? GIN : entries_in_flight<float, VPT, MINB>();
  constexpr bool PFY = !(OPT & 2);
  constexpr int RPB = kBlock / TPR;
  constexpr int PF = TPR == 1 ? G : 1;
  const int sub = threadIdx.x % TPR;
  const int grp = threadIdx.x / TPR;
  const unsigned mask = 0xffffffffu;
  constexpr bool SMD = DOTS && (OPT & 8);
  extern __shared__ double real_sdots[];  // [2][VPT][kBlock] with SMD
  double d_nn[DOTS && !SMD ? VPT : 1], d_np[DOTS && !SMD ? VPT : 1];
  if constexpr (DOTS && !SMD) {
#pragma unroll
    for (int j = 0; j < VPT; j++) d_nn[j] = d_np[j] = 0.0;
  }
  if constexpr (SMD) {
#pragma unroll
    for (int j = 0; j < 2 * VPT; j++) real_sdots[j * kBlock + threadIdx.x] = 0.0;
  }
  // slice bounds a tile ahead of the entries for thread shares below 32 B
  // (for (8, 8) loading them with the entries measured 3% faster)
  constexpr bool PB = sizeof(float) * VPT < 32 && !(OPT & 1);
  const uint64_t ntiles = ((uint64_t)A.nslices * 32 + RPB - 1) / RPB;
  RRowFetch<TPR, VPT, PF> cur, nxt;
  RowBounds bn{0, 0};
  if (blockIdx.x < ntiles)
    rfetch_row<TPR, VPT, PF, FIRST, PFY>(A, Bp, y, blockIdx.x, grp, sub,
                                         load_bounds<TPR>(A, blockIdx.x, grp), cur);
  if constexpr (PB)
    if (blockIdx.x + gridDim.x < ntiles) bn = load_bounds<TPR>(A, blockIdx.x + gridDim.x, grp);
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint64_t tnext = tile + gridDim.x, tnext2 = tnext + gridDim.x;
    RowBounds bn2{0, 0};
    if constexpr (PB) {
      if (tnext < ntiles)
        rfetch_row<TPR, VPT, PF, FIRST, PFY>(A, Bp, y, tnext, grp, sub, bn, nxt);
      if (tnext2 < ntiles) bn2 = load_bounds<TPR>(A, tnext2, grp);
    } else {
      if (tnext < ntiles)
        rfetch_row<TPR, VPT, PF, FIRST, PFY>(A, Bp, y, tnext, grp, sub,
                                             load_bounds<TPR>(A, tnext, grp), nxt);
    }
    if (cur.ok) {
      const uint32_t row = cur.row, l = cur.l, cb = cur.cb, w = cur.ce - cur.cb;
      double acc[VPT];
      if constexpr (FIRST) {
#pragma unroll
        for (int j = 0; j < VPT; j++) acc[j] = 0.0;
      } else if constexpr (PFY) {
#pragma unroll
        for (int j = 0; j < VPT; j++) acc[j] = cur.live ? -(double)P::getf(cur.yr, j) : 0.0;
      } else {
        L yv[NL];
        if (cur.live) P::load_rw(y + (uint64_t)row * Bp, sub, yv);
#pragma unroll
        for (int j = 0; j < VPT; j++) acc[j] = cur.live ? -(double)P::getf(yv, j) : 0.0;
      }
      if constexpr (TPR == 1) {
        for (uint32_t kb = 0; kb < w; kb += G) {
          uint32_t cc[G];
          double vv[G];
          L raw[G][NL];
#pragma unroll
          for (int g = 0; g < G; g++)
            cc[g] = kb == 0 ? cur.cc[g]
                            : ((kb + g < w) ? __ldcs(A.col + (uint64_t)(cb + kb + g) * 32 + l) : kPad);
#pragma unroll
          for (int g = 0; g < G; g++)
            if (cc[g] != kPad) {
              vv[g] = __ldcs(A.vre + (uint64_t)(cb + kb + g) * 32 + l);
              P::load(x + (uint64_t)cc[g] * Bp, sub, raw[g]);
            }
#pragma unroll
          for (int g = 0; g < G; g++) {
            if (cc[g] == kPad) continue;
            double v = vv[g];
            if constexpr (FIRST) v = v * 0.5;
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = fma(v, (double)P::getf(raw[g], j), acc[j]);
          }
        }
      } else {
        for (uint32_t kb = 0; kb < w; kb += TPR) {
          uint32_t myc;
          double myv;
          if (kb == 0) {
            myc = cur.cc[0];
            myv = cur.vv[0];
          } else {
            myc = kPad;
            myv = 0.0;
            if (kb + sub < w) {
              myc = __ldcs(A.col + (uint64_t)(cb + kb + sub) * 32 + l);
              if (myc != kPad) myv = __ldcs(A.vre + (uint64_t)(cb + kb + sub) * 32 + l);
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
              double v = __shfl_sync(mask, myv, (int)min(j0 + g, nk - 1), TPR);
              if (cc[g] == kPad) continue;
              if constexpr (FIRST) v = v * 0.5;
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[j] = fma(v, (double)P::getf(raw[g], j), acc[j]);
            }
          }
        }
      }
      if (cur.live) {
        if (target_hit(tg, row)) {
          for (uint32_t i = target_first(tg, row); i < tg.count && __ldg(tg.row + i) == row; i++) {
            const int jt = P::slot_of(sub, __ldg(tg.col + i));
            if (jt >= 0) {
#pragma unroll
              for (int j = 0; j < VPT; j++)
                if (j == jt)
                  tg.mu[(uint64_t)__ldg(tg.out + i) * tg.ld + n_out] = make_double2(acc[j], 0.0);
            }
          }
        }
        float af[VPT];
#pragma unroll
        for (int j = 0; j < VPT; j++) af[j] = __double2float_rn(acc[j]);
        P::storef(y + (uint64_t)row * Bp, sub, af);
        if constexpr (DOTS) {
          // the complex64 kernel's terms with zero imaginary parts
          L self[NL];
          P::load(x + (uint64_t)row * Bp, sub, self);
#pragma unroll
          for (int j = 0; j < VPT; j++) {
            const float b = P::getf(self, j);
            if constexpr (SMD) {
              real_sdots[j * kBlock + threadIdx.x] += (double)fmaf(af[j], af[j], 0.0f);
              real_sdots[(VPT + j) * kBlock + threadIdx.x] += (double)fmaf(af[j], b, 0.0f);
            } else {
              d_nn[j] += (double)fmaf(af[j], af[j], 0.0f);
              d_np[j] += (double)fmaf(af[j], b, 0.0f);
            }
          }
        }
      }
    }
    cur = nxt;
    bn = bn2;
  }
  if constexpr (DOTS) {
    __shared__ double red[kBlock][2];
#pragma unroll 1
    for (int j = 0; j < VPT; j++) {
      if constexpr (SMD) {
        red[threadIdx.x][0] = real_sdots[j * kBlock + threadIdx.x];
        red[threadIdx.x][1] = real_sdots[(VPT + j) * kBlock + threadIdx.x];
      } else {
        red[threadIdx.x][0] = d_nn[j];
        red[threadIdx.x][1] = d_np[j];
      }
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

// Sets x[from_b][b] = 1 for each source (x zeroed beforehand) and the zeroth
// moments, as kpm_init_sources.
static __global__ void kpm_init_sources_real(uint32_t B, uint32_t Bp, const uint32_t *from,
                                             float *x, Targets tg) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B) x[(uint64_t)from[i] * Bp + i] = 1.0f;
  if (i < tg.count) {
    const uint32_t b = tg.col[i];
    const double v = (tg.row[i] == from[b]) ? 1.0 : 0.0;
    tg.mu[(uint64_t)tg.out[i] * tg.ld] = make_double2(v, 0.0);
  }
}

}  // namespace tbtkkpm
