// Multi-model recursion step on real float vectors: kpm_multi_step for
// models whose Hamiltonian is real (see kpm_real.cuh for why the real step
// gives the complex64 step's values).  A model's vec[] buffers then hold
// [rows][W] floats; the lane, target, moment and fixed-point-sum handling is
// kpm_multi_step's, with the dot-product terms of real values.
#pragma once

#include "kpm_multi.cuh"
#include "kpm_real.cuh"

namespace tbtkkpm {

template <int TPR, int VPT, int MINB>
__global__ void __launch_bounds__(kBlock, MINB)
kpm_multi_step_real(const MultiModel *__restrict__ models, const MultiHeader *__restrict__ hdr,
                    uint32_t step_offset, uint32_t W, uint32_t ld) {
  using P = RPack<TPR, VPT>;
  using L = typename P::L;
  constexpr int NL = P::NL;
  constexpr int G = entries_in_flight<float, VPT, MINB>();
  constexpr int PF = TPR == 1 ? G : 1;
  const int sub = threadIdx.x % TPR;
  const int grp = threadIdx.x / TPR;
  const unsigned mask = 0xffffffffu;
  const uint32_t nmodels = hdr->nmodels, total = hdr->total_tiles;
  const uint32_t *__restrict__ tile_model = hdr->tile_model;
  const int32_t n = multi_step_index(hdr, step_offset);
  if (nmodels == 0) return;

  // per-thread fixed-point sums, [2 * VPT][kBlock] in dynamic shared memory
  // (64 KB at 16 values per thread, above the static limit)
  extern __shared__ long long mreal_sums[];
  long long (*msum)[kBlock] = reinterpret_cast<long long (*)[kBlock]>(mreal_sums);
#pragma unroll
  for (int j = 0; j < 2 * VPT; j++) msum[j][threadIdx.x] = 0;

  uint32_t mi = kPad, fi = kPad;
  Sell A{}, FA{};
  const float *x = nullptr;
  float *y = nullptr;
  const float *fy = nullptr;
  uint32_t ft0 = 0;
  uint32_t first = 0;
  const uint32_t *t_bitmap = nullptr, *t_row = nullptr, *t_col = nullptr;
  const int32_t *t_base = nullptr;
  long long *t_dots = nullptr;
  uint32_t t_count = 0;

  auto bounds_of = [&](uint32_t t, uint32_t &model) -> RowBounds {
    model = __ldg(tile_model + t);
    const MultiModel *q = models + model;
    Sell s{};
    s.slice_ptr = q->A.slice_ptr;
    s.nslices = q->A.nslices;
    return load_bounds<TPR>(s, t - q->tile0, grp);
  };
  auto fetch = [&](uint32_t t, uint32_t i, RowBounds b, RRowFetch<TPR, VPT, PF> &f) {
    if (i != fi) {
      fi = i;
      const MultiModel *q = models + i;
      FA.slice_ptr = q->A.slice_ptr;
      FA.col = q->A.col;
      FA.vre = q->A.vre;
      FA.N = q->A.N;
      FA.nslices = q->A.nslices;
      fy = reinterpret_cast<const float *>(q->vec[n & 1]);
      ft0 = q->tile0;
    }
    rfetch_row<TPR, VPT, PF, false>(FA, W, fy, t - ft0, grp, sub, b, f);
  };
  auto next_tile = [&](uint32_t t) -> uint32_t {
    const uint32_t nt = t + 1;
    if (nt % kRun != 0) return nt;
    return (t / kRun + gridDim.x) * kRun;
  };

  RRowFetch<TPR, VPT, PF> cur, nxt;
  uint32_t cur_model = 0, nxt_model = 0;
  uint32_t w = blockIdx.x * kRun;
  if (w < total) {
    const RowBounds b0 = bounds_of(w, cur_model);
    fetch(w, cur_model, b0, cur);
  }
  uint32_t wn = next_tile(w), bm = 0;
  RowBounds bb{0, 0};
  if (wn < total) bb = bounds_of(wn, bm);
  for (; w < total; w = wn, wn = next_tile(wn)) {
    if (cur_model != mi) {
      if (mi != kPad) multi_flush<P, VPT, TPR>(msum, t_dots, W, sub);
      mi = cur_model;
      const MultiModel *md = models + mi;
      A.slice_ptr = md->A.slice_ptr;
      A.col = md->A.col;
      A.vre = md->A.vre;
      A.N = md->A.N;
      A.nslices = md->A.nslices;
      x = reinterpret_cast<const float *>(md->vec[(n + 1) & 1]);
      y = reinterpret_cast<float *>(md->vec[n & 1]);
      t_bitmap = md->bitmap;
      t_row = md->trow;
      t_col = md->tcol;
      t_count = md->tcount;
      t_base = md->base;
      t_dots = md->dots;
      first = 0;
#pragma unroll
      for (int j = 0; j < VPT; j++)
        if (n - __ldg(t_base + P::col_of(sub, j)) == 1) first |= 1u << j;
    }
    if (wn < total) {
      fetch(wn, bm, bb, nxt);
      nxt_model = bm;
    }
    const uint32_t wn2 = next_tile(wn);
    if (wn2 < total) bb = bounds_of(wn2, bm);
    if (cur.ok) {
      const uint32_t row = cur.row, l = cur.l, cb = cur.cb, wd = cur.ce - cur.cb;
      double acc[VPT];
#pragma unroll
      for (int j = 0; j < VPT; j++)
        acc[j] = ((first >> j) & 1u) ? 0.0 : (cur.live ? -(double)P::getf(cur.yr, j) : 0.0);
      if constexpr (TPR == 1) {
        for (uint32_t kb = 0; kb < wd; kb += G) {
          uint32_t cc[G];
          double vv[G];
          L raw[G][NL];
#pragma unroll
          for (int g = 0; g < G; g++)
            cc[g] = kb == 0 ? cur.cc[g]
                            : ((kb + g < wd) ? __ldcs(A.col + (uint64_t)(cb + kb + g) * 32 + l) : kPad);
#pragma unroll
          for (int g = 0; g < G; g++)
            if (cc[g] != kPad) {
              vv[g] = __ldcs(A.vre + (uint64_t)(cb + kb + g) * 32 + l);
              P::load(x + (uint64_t)cc[g] * W, sub, raw[g]);
            }
#pragma unroll
          for (int g = 0; g < G; g++) {
            if (cc[g] == kPad) continue;
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = fma(vv[g], (double)P::getf(raw[g], j), acc[j]);
          }
        }
      } else {
        for (uint32_t kb = 0; kb < wd; kb += TPR) {
          uint32_t myc;
          double myv;
          if (kb == 0) {
            myc = cur.cc[0];
            myv = cur.vv[0];
          } else {
            myc = kPad;
            myv = 0.0;
            if (kb + sub < wd) {
              myc = __ldcs(A.col + (uint64_t)(cb + kb + sub) * 32 + l);
              if (myc != kPad) myv = __ldcs(A.vre + (uint64_t)(cb + kb + sub) * 32 + l);
            }
          }
          const uint32_t nk = min((uint32_t)TPR, wd - kb);
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
              if (cc[g] != kPad) P::load(x + (uint64_t)cc[g] * W, sub, raw[g]);
#pragma unroll
            for (int g = 0; g < G; g++) {
              const double v = __shfl_sync(mask, myv, (int)min(j0 + g, nk - 1), TPR);
              if (cc[g] == kPad) continue;
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[j] = fma(v, (double)P::getf(raw[g], j), acc[j]);
            }
          }
        }
      }
      if (cur.live) {
#pragma unroll
        for (int j = 0; j < VPT; j++)
          if ((first >> j) & 1u) acc[j] = acc[j] * 0.5;
        if ((__ldg(t_bitmap + (row >> 5)) >> (row & 31)) & 1u) {
          uint32_t lo = 0, hi = t_count;
          while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(t_row + mid) < row) lo = mid + 1; else hi = mid;
          }
          for (uint32_t i = lo; i < t_count && __ldg(t_row + i) == row; i++) {
            const uint32_t tc = __ldg(t_col + i);
            const uint32_t c = tc & kLaneBits;
            const int jt = P::slot_of(sub, c);
            if (jt < 0) continue;
            double2 *dst = multi_target_dst(models + mi, tc, n - __ldg(t_base + c), ld);
            if (dst) {
#pragma unroll
              for (int j = 0; j < VPT; j++)
                if (j == jt) *dst = make_double2(acc[j], 0.0);
            }
          }
        }
        float af[VPT];
#pragma unroll
        for (int j = 0; j < VPT; j++) af[j] = __double2float_rn(acc[j]);
        P::storef(y + (uint64_t)row * W, sub, af);
        L self[NL];
        P::load(x + (uint64_t)row * W, sub, self);
#pragma unroll
        for (int j = 0; j < VPT; j++) {
          const float b = P::getf(self, j);
          msum[j][threadIdx.x] += __float2ll_rn(fmaf(af[j], af[j], 0.0f) * kFixScale);
          msum[VPT + j][threadIdx.x] += __float2ll_rn(fmaf(af[j], b, 0.0f) * kFixScale);
        }
      }
    }
    cur = nxt;
    cur_model = nxt_model;
  }
  if (mi != kPad) multi_flush<P, VPT, TPR>(msum, t_dots, W, sub);
}

template <int TPR, int VPT, int MINB>
void launch_multi_real(cudaStream_t st, int device, const MultiModel *models,
                       const MultiHeader *hdr, uint32_t step_offset, uint32_t W, uint32_t ld,
                       const MultiLaunch &) {
  auto kern = kpm_multi_step_real<TPR, VPT, MINB>;
  constexpr uint32_t smem = 2u * VPT * kBlock * 8u;
  static int per_sm[64] = {0};
  const int d = device & 63;
  if (per_sm[d] == 0) {
    if (smem > 48u * 1024u)
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kBlock, smem) != cudaSuccess ||
        nb < 1) {
      cudaGetLastError();
      nb = 1;
    }
    per_sm[d] = nb;
  }
  kern<<<(unsigned)(per_sm[d] * sm_count(device)), kBlock, smem, st>>>(models, hdr, step_offset,
                                                                       W, ld);
}

#define TBTKKPM_MULTI_REAL_ENTRY(T, P, MB) {T, P, MB, &launch_multi_real<T, P, MB>}

extern const MultiEntry kMultiStepsReal[];
extern const int kNumMultiStepsReal;

}  // namespace tbtkkpm
