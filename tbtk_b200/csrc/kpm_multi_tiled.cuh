// Tile-staged multi-model recursion step: the server's step over every model
// with busy lanes, with the gathered rows of each tile staged in shared
// memory by bulk copies (the single-model kpm_step_tiled, generalised to a
// launch whose tiles belong to different models).
//
// A launch covers one lane class (lane width W, real or complex vectors).
// Every model of the class has a gather plan for R-row tiles (the matrix
// handle's plan, k_plan_fill in kpm_tiled.cuh); kpm_multi_tilemap_tiled
// writes, per launch tile, its model and its plan header with the runs
// rebased into one run list of the launch.  Warp 0 of a block is the
// producer: for each tile of the block's sequence it copies the tile's
// entries (values and shared-memory slots), its own rows of j_n and j_{n-1}
// and the runs of outside rows of j_n into a ring stage.  Warps 1..CW
// compute the tile's rows from shared memory with the per-element
// arithmetic of kpm_multi_step / kpm_multi_step_real (acc = -j_{n-1}, or 0
// for a lane at its local step 1, FMAs in CSR entry order, the first step
// halved exactly, one rounding to float), so stored vectors and moments are
// the register-staged kernels' bit for bit; the doubling sums are the same
// fixed-point terms, kept per thread in registers and added into the
// model's sums with one atomic per column and warp when the warp changes
// model.
//
// Only non-multicast bulk copies from this GPU's memory are issued.  Every
// mbarrier wait is bounded (`wait_limit` polls): a wait that runs out sets
// *err and ends the loops, and before the block exits every copy it issued
// has landed (waited for with the library's bound kWaitLimit).
#pragma once

#include "kpm_multi.cuh"
#include "kpm_tiled.cuh"

namespace tbtkkpm {

// Tile-staged variant code of a multi-model entry: kTiledVariant + 1000*R +
// 10*CW + BPS (R rows per tile, CW consumer warps, BPS blocks per SM).
constexpr int kMultiTiledVariant = 100000;
inline bool is_multi_tiled(int minb) { return minb >= kMultiTiledVariant; }
inline int multi_tiled_rows(int minb) { return ((minb - kMultiTiledVariant) % 1000000) / 1000; }
inline int multi_tiled_bps(int minb) { return minb % 10; }

// Per launch tile: its model and its plan header, the runs copied into the
// launch's run list at the model's run0.  One block per model.
static __global__ void kpm_multi_tilemap_tiled(const MultiModel *__restrict__ models,
                                               const MultiHeader *__restrict__ hdr,
                                               uint32_t *tile_model, uint4 *tile_hdr,
                                               uint2 *tile_runs) {
  if (blockIdx.x >= hdr->nmodels) return;
  const MultiModel &q = models[blockIdx.x];
  const uint32_t t0 = q.tile0, nt = q.ntiles, r0 = q.run0;
  for (uint32_t t = threadIdx.x; t < nt; t += blockDim.x) {
    uint4 h = q.p_hdr[t];
    h.y += r0;
    tile_model[t0 + t] = blockIdx.x;
    tile_hdr[t0 + t] = h;
  }
  for (uint32_t k = threadIdx.x; k < q.p_nruns; k += blockDim.x) tile_runs[r0 + k] = q.p_runs[k];
}

template <bool CPLX, int TPR, int VPT, int R, int CW, int BPS>
__global__ void __launch_bounds__(32 * (CW + 1), BPS)
kpm_multi_tiled(const MultiModel *__restrict__ models, const MultiHeader *__restrict__ hdr,
                TiledLayout LY, uint32_t step_offset, uint32_t W, uint32_t ld, int *err,
                uint32_t wait_limit) {
  using E = typename TiledTypes<CPLX>::E;
  using Val = typename TiledTypes<CPLX>::Val;
  using Pk = typename std::conditional<CPLX, Pack<float2, TPR, VPT>, RPack<TPR, VPT>>::type;
  using L = typename Pk::L;
  constexpr int NL = Pk::NL;
  constexpr int RPP = CW * 32 / TPR;  // rows per pass
  constexpr int PASSES = (R + RPP - 1) / RPP;
  static_assert(CW * 32 % TPR == 0, "a row group must divide the consumer threads");
  extern __shared__ __align__(128) unsigned char tsm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(tsm);
  uint64_t *empty = full + kTiledMaxStages;
  unsigned char *ring = tsm + kTiledHeader;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t S = LY.stages;
  const uint32_t rowbytes = W * (uint32_t)sizeof(E);
  const uint32_t total = hdr->total_tiles;
  const uint32_t *__restrict__ tile_model = hdr->tile_model;
  const uint4 *__restrict__ thdr = hdr->tile_hdr;
  const uint2 *__restrict__ truns = hdr->tile_runs;
  const int32_t n = hdr->n_base + (int32_t)step_offset;
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], CW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // the block's i-th tile: runs of kRun consecutive tiles, run b, b + grid, ...
  auto tile_at = [&](uint32_t i) -> uint32_t {
    return (blockIdx.x + (i / kRun) * gridDim.x) * kRun + i % kRun;
  };

  if (warp == 0) {
    // ---------------------------------------------------------- producer
    // Tile i is copied into stage i % S.  Headers and models two tiles
    // ahead and the first 32 runs one tile ahead keep the dependent loads
    // off the issue path; a model's pointers are reloaded when it changes.
    uint32_t t0 = tile_at(0), t1 = tile_at(1);
    uint4 h0 = make_uint4(0, 0, 0, 0), h1 = h0;
    uint32_t q0 = 0, q1 = 0;
    if (t0 < total) {
      h0 = __ldg(thdr + t0);
      q0 = __ldg(tile_model + t0);
    }
    if (t1 < total) {
      h1 = __ldg(thdr + t1);
      q1 = __ldg(tile_model + t1);
    }
    uint2 run0 = make_uint2(0, 0);
    if (t0 < total && (uint32_t)lane < (h0.w >> 16)) run0 = __ldg(truns + h0.y + lane);
    uint32_t cq = kPad;
    const Val *m_val = nullptr;
    const uint16_t *m_slot = nullptr;
    const E *m_x = nullptr, *m_y = nullptr;
    uint32_t m_t0 = 0, m_N = 0;
    bool failed = false;
    uint32_t issued = 0;
    for (uint32_t i = 0; t0 < total; i++) {
      const uint32_t t2 = tile_at(i + 2);
      uint4 h2 = make_uint4(0, 0, 0, 0);
      uint32_t q2 = 0;
      if (t2 < total) {
        h2 = __ldg(thdr + t2);
        q2 = __ldg(tile_model + t2);
      }
      uint2 run1 = make_uint2(0, 0);
      if (t1 < total && (uint32_t)lane < (h1.w >> 16)) run1 = __ldg(truns + h1.y + lane);
      if (q0 != cq) {
        cq = q0;
        const MultiModel *md = models + q0;
        m_val = static_cast<const Val *>(md->p_val);
        m_slot = md->p_slot;
        m_x = reinterpret_cast<const E *>(md->vec[(n + 1) & 1]);
        m_y = reinterpret_cast<const E *>(md->vec[n & 1]);
        m_t0 = md->tile0;
        m_N = md->A.N;
      }
      const uint32_t s = i % S;
      if (i >= S && !mbar_wait_limit(&empty[s], ((i / S) - 1) & 1u, wait_limit)) {
        failed = true;
        break;
      }
      unsigned char *st = ring + (size_t)s * LY.stage_bytes;
      const uint32_t w = h0.w & 0xffffu, nruns = h0.w >> 16, nuniq = h0.z;
      const uint32_t r0 = (t0 - m_t0) * R, Rt = min((uint32_t)R, m_N - r0);
      const uint32_t ebytes = w * R * (uint32_t)sizeof(Val), sbytes = w * R * 2u;
      const uint32_t bytes = (w ? ebytes + sbytes : 0u) + (2 * Rt + nuniq) * rowbytes;
      if (lane == 0) mbar_expect_tx(&full[s], bytes);
      __syncwarp();
      const uint64_t e0 = (uint64_t)h0.x * R;
      if (w) {
        if (lane == 0) bulk_load(st, m_val + e0, ebytes, &full[s]);
        if (lane == 1) bulk_load(st + LY.off_slots, m_slot + e0, sbytes, &full[s]);
      }
      if (lane == 2) bulk_load(st + LY.off_xs, m_x + (uint64_t)r0 * W, Rt * rowbytes, &full[s]);
      if (lane == 3) bulk_load(st + LY.off_prev, m_y + (uint64_t)r0 * W, Rt * rowbytes, &full[s]);
      for (uint32_t c = 0; c < nruns; c += 32) {
        uint2 rn = run0;
        if (c > 0) rn = (c + lane < nruns) ? __ldg(truns + h0.y + c + lane) : make_uint2(0, 0);
        if (c + lane < nruns) {
          const uint32_t slot = R + (rn.y >> 16), len = rn.y & 0xffffu;
          bulk_load(st + LY.off_xs + (size_t)slot * rowbytes, m_x + (uint64_t)rn.x * W,
                    len * rowbytes, &full[s]);
        }
      }
      issued = i + 1;
      t0 = t1;
      h0 = h1;
      q0 = q1;
      run0 = run1;
      t1 = t2;
      h1 = h2;
      q1 = q2;
    }
    if (failed && lane == 0) atomicExch(err, kErrTimeout);
    // every copy issued into this block's ring lands (or its wait runs out)
    // before the block exits
    if (lane == 0)
      for (uint32_t s = 0; s < S && s < issued; s++) {
        const uint32_t fills = (issued - 1 - s) / S + 1;
        if (!mbar_wait_limit(&full[s], (fills - 1) & 1u, kWaitLimit)) atomicExch(err, kErrTimeout);
      }
  } else {
    // ---------------------------------------------------------- consumers
    const int ct = threadIdx.x - 32;
    const int sub = ct % TPR, grp = ct / TPR;
    uint32_t cq = kPad;
    const uint32_t *t_bitmap = nullptr, *t_row = nullptr, *t_col = nullptr;
    const int32_t *t_base = nullptr;
    long long *t_dots = nullptr;
    uint32_t t_count = 0, m_t0 = 0, m_N = 0, first = 0;
    E *m_y = nullptr;
    long long s_nn[VPT], s_np[VPT];
#pragma unroll
    for (int j = 0; j < VPT; j++) s_nn[j] = s_np[j] = 0;
    // the warp's sums over threads of the same columns, one atomic per
    // column and warp (warp-uniform: the warp's threads share the tile)
    auto flush = [&]() {
#pragma unroll
      for (int j = 0; j < VPT; j++) {
        long long a = s_nn[j], b = s_np[j];
#pragma unroll
        for (int off = TPR; off < 32; off <<= 1) {
          a += __shfl_xor_sync(0xffffffffu, a, off);
          b += __shfl_xor_sync(0xffffffffu, b, off);
        }
        if (lane < TPR) {
          const uint32_t c = Pk::col_of(sub, j);
          if (a) atomicAdd(reinterpret_cast<unsigned long long *>(t_dots + c), (unsigned long long)a);
          if (b) atomicAdd(reinterpret_cast<unsigned long long *>(t_dots + W + c), (unsigned long long)b);
        }
        s_nn[j] = s_np[j] = 0;
      }
    };
    bool failed = false;
    for (uint32_t i = 0;; i++) {
      const uint32_t t = tile_at(i);
      if (t >= total) break;
      const uint32_t s = i % S;
      const uint32_t q = __ldg(tile_model + t);
      const uint32_t w = __ldg(thdr + t).w & 0xffffu;
      if (q != cq) {
        if (cq != kPad) flush();
        cq = q;
        const MultiModel *md = models + q;
        t_bitmap = md->bitmap;
        t_row = md->trow;
        t_col = md->tcol;
        t_count = md->tcount;
        t_base = md->base;
        t_dots = md->dots;
        m_t0 = md->tile0;
        m_N = md->A.N;
        m_y = reinterpret_cast<E *>(md->vec[n & 1]);
        first = 0;
#pragma unroll
        for (int j = 0; j < VPT; j++)
          if (n - __ldg(t_base + Pk::col_of(sub, j)) == 1) first |= 1u << j;
      }
      const uint32_t r0 = (t - m_t0) * R, Rt = min((uint32_t)R, m_N - r0);
      uint32_t bw[PASSES];
#pragma unroll
      for (int p = 0; p < PASSES; p++) {
        const uint32_t lr = grp + p * RPP;
        bw[p] = lr < Rt ? __ldg(t_bitmap + ((r0 + lr) >> 5)) : 0u;
      }
      if (!mbar_wait_limit(&full[s], (i / S) & 1u, wait_limit)) {
        failed = true;
        break;
      }
      const unsigned char *st = ring + (size_t)s * LY.stage_bytes;
      const Val *vals = reinterpret_cast<const Val *>(st);
      const uint16_t *slots = reinterpret_cast<const uint16_t *>(st + LY.off_slots);
      const E *xs = reinterpret_cast<const E *>(st + LY.off_xs);
      const E *prev = reinterpret_cast<const E *>(st + LY.off_prev);
#pragma unroll
      for (int p = 0; p < PASSES; p++) {
        const uint32_t lr = grp + p * RPP;
        if (lr >= Rt) continue;
        const uint32_t row = r0 + lr;
        if constexpr (CPLX) {
          double2 acc[VPT];
          {
            L yv[NL];
            Pk::load_rw(reinterpret_cast<const float2 *>(prev) + (size_t)lr * W, sub, yv);
#pragma unroll
            for (int j = 0; j < VPT; j++) {
              const double2 f = Pk::get(yv, j);
              acc[j] = ((first >> j) & 1u) ? make_double2(0.0, 0.0) : make_double2(-f.x, -f.y);
            }
          }
          for (uint32_t k = 0; k < w; k++) {
            const uint16_t sl = slots[k * R + lr];
            if (sl == kSlotPad) break;
            const double2 v = vals[k * R + lr];
            L xr[NL];
            Pk::load_rw(reinterpret_cast<const float2 *>(xs) + (size_t)sl * W, sub, xr);
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = cmac<false>(acc[j], v, Pk::get(xr, j));
          }
#pragma unroll
          for (int j = 0; j < VPT; j++)
            if ((first >> j) & 1u) acc[j] = make_double2(acc[j].x * 0.5, acc[j].y * 0.5);
          if ((bw[p] >> (row & 31)) & 1u) {
            uint32_t lo = 0, hi = t_count;
            while (lo < hi) {
              const uint32_t mid = (lo + hi) >> 1;
              if (__ldg(t_row + mid) < row) lo = mid + 1; else hi = mid;
            }
            for (uint32_t e = lo; e < t_count && __ldg(t_row + e) == row; e++) {
              const uint32_t tc = __ldg(t_col + e);
              const uint32_t c = tc & kLaneBits;
              const int jt = Pk::slot_of(sub, c);
              if (jt < 0) continue;
              double2 *dst = multi_target_dst(models + cq, tc, n - __ldg(t_base + c), ld);
              if (dst) {
#pragma unroll
                for (int j = 0; j < VPT; j++)
                  if (j == jt) *dst = acc[j];
              }
            }
          }
          float2 af[VPT];
#pragma unroll
          for (int j = 0; j < VPT; j++)
            af[j] = make_float2(__double2float_rn(acc[j].x), __double2float_rn(acc[j].y));
          Pk::storef(reinterpret_cast<float2 *>(m_y) + (uint64_t)row * W, sub, af);
          L self[NL];
          Pk::load_rw(reinterpret_cast<const float2 *>(xs) + (size_t)lr * W, sub, self);
#pragma unroll
          for (int j = 0; j < VPT; j++) {
            const float2 b = Pk::getf(self, j);
            s_nn[j] += __float2ll_rn(fmaf(af[j].x, af[j].x, af[j].y * af[j].y) * kFixScale);
            s_np[j] += __float2ll_rn(fmaf(af[j].x, b.x, af[j].y * b.y) * kFixScale);
          }
        } else {
          double acc[VPT];
          {
            L yv[NL];
            Pk::load_rw(reinterpret_cast<const float *>(prev) + (size_t)lr * W, sub, yv);
#pragma unroll
            for (int j = 0; j < VPT; j++)
              acc[j] = ((first >> j) & 1u) ? 0.0 : -(double)Pk::getf(yv, j);
          }
          for (uint32_t k = 0; k < w; k++) {
            const uint16_t sl = slots[k * R + lr];
            if (sl == kSlotPad) break;
            const double v = vals[k * R + lr];
            L xr[NL];
            Pk::load_rw(reinterpret_cast<const float *>(xs) + (size_t)sl * W, sub, xr);
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = fma(v, (double)Pk::getf(xr, j), acc[j]);
          }
#pragma unroll
          for (int j = 0; j < VPT; j++)
            if ((first >> j) & 1u) acc[j] = acc[j] * 0.5;
          if ((bw[p] >> (row & 31)) & 1u) {
            uint32_t lo = 0, hi = t_count;
            while (lo < hi) {
              const uint32_t mid = (lo + hi) >> 1;
              if (__ldg(t_row + mid) < row) lo = mid + 1; else hi = mid;
            }
            for (uint32_t e = lo; e < t_count && __ldg(t_row + e) == row; e++) {
              const uint32_t tc = __ldg(t_col + e);
              const uint32_t c = tc & kLaneBits;
              const int jt = Pk::slot_of(sub, c);
              if (jt < 0) continue;
              double2 *dst = multi_target_dst(models + cq, tc, n - __ldg(t_base + c), ld);
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
          Pk::storef(reinterpret_cast<float *>(m_y) + (uint64_t)row * W, sub, af);
          L self[NL];
          Pk::load_rw(reinterpret_cast<const float *>(xs) + (size_t)lr * W, sub, self);
#pragma unroll
          for (int j = 0; j < VPT; j++) {
            const float b = Pk::getf(self, j);
            s_nn[j] += __float2ll_rn(fmaf(af[j], af[j], 0.0f) * kFixScale);
            s_np[j] += __float2ll_rn(fmaf(af[j], b, 0.0f) * kFixScale);
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
    if (cq != kPad) flush();
    if (failed && lane == 0) atomicExch(err, kErrTimeout);
  }
}

// Grid: BPS blocks per SM.  Launches nothing when the class has no layout
// (ly.stages == 0: the host falls back to a register-staged entry).
template <bool CPLX, int TPR, int VPT, int R, int CW, int BPS>
void launch_multi_tiled(cudaStream_t st, int device, const MultiModel *models,
                        const MultiHeader *hdr, uint32_t step_offset, uint32_t W, uint32_t ld,
                        const MultiLaunch &ml) {
  auto kern = kpm_multi_tiled<CPLX, TPR, VPT, R, CW, BPS>;
  if (ml.ly.stages == 0) return;
  static bool attr[64] = {false};
  const int d = device & 63;
  if (!attr[d]) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tiled_budget(BPS));
    attr[d] = true;
  }
  const uint32_t smem = kTiledHeader + ml.ly.stages * ml.ly.stage_bytes;
  kern<<<(unsigned)(BPS * sm_count(device)), 32 * (CW + 1), smem, st>>>(
      models, hdr, ml.ly, step_offset, W, ld, ml.err, ml.wait_limit);
}

#define TBTKKPM_MULTI_TILED_ENTRY(CPLX, T, P, R, CW, BPS) \
  {T, P, kMultiTiledVariant + 1000 * R + 10 * CW + BPS, &launch_multi_tiled<CPLX, T, P, R, CW, BPS>}

extern const MultiEntry kMultiTiled[];
extern const int kNumMultiTiled;
extern const MultiEntry kMultiTiledReal[];
extern const int kNumMultiTiledReal;

}  // namespace tbtkkpm
