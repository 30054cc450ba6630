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

// Tile-staged variant code of a multi-model entry: kTiledVariant +
// 1000000*CV + 1000*R + 10*CW + BPS (CV the widening split, R rows per tile,
// CW consumer warps, BPS blocks per SM).
constexpr int kMultiTiledVariant = 100000;
inline bool is_multi_tiled(int minb) { return minb >= kMultiTiledVariant; }
inline int multi_tiled_rows(int minb) { return ((minb - kMultiTiledVariant) % 1000000) / 1000; }
inline int multi_tiled_bps(int minb) { return minb % 10; }

// Descriptor of a launch tile, 6 x 16 bytes: [0] its plan header {entry
// chunk, first run in the launch's run list, distinct outside rows, w |
// runs << 16}; [1] {model | rows << 16, first row, target bits of its rows
// (2 words)}; [2..5] its first kDescRuns runs.  The targets change only
// between ticks, so one map serves every step of a tick.
constexpr uint32_t kDescWords = 6;  // uint4 per descriptor
constexpr uint32_t kDescRuns = 8;

// Writes the descriptors (and the launch's run list) of every tile of the
// launch's models: one block per model; R rows per tile (R divides 64).
static __global__ void kpm_multi_tilemap_tiled(const MultiModel *__restrict__ models,
                                               const MultiHeader *__restrict__ hdr, uint32_t R,
                                               uint4 *tile_desc, uint2 *tile_runs) {
  if (blockIdx.x >= hdr->nmodels) return;
  const MultiModel &q = models[blockIdx.x];
  const uint32_t t0 = q.tile0, nt = q.ntiles, ro = q.run0, N = q.A.N;
  for (uint32_t t = threadIdx.x; t < nt; t += blockDim.x) {
    const uint4 h = q.p_hdr[t];
    uint4 *d = tile_desc + (size_t)(t0 + t) * kDescWords;
    d[0] = make_uint4(h.x, h.y + ro, h.z, h.w);
    const uint32_t r0 = t * R, rt = min(R, N - r0);
    // bits of rows r0 .. r0 + rt - 1 (r0 a multiple of R)
    unsigned long long bits = 0;
    for (uint32_t w = r0 >> 5; w <= (r0 + rt - 1) >> 5; w++)
      bits |= (unsigned long long)q.bitmap[w] << (32 * (w - (r0 >> 5)));
    bits >>= (r0 & 31);
    if (rt < 64) bits &= (1ull << rt) - 1;
    d[1] = make_uint4(blockIdx.x | (rt << 16), r0, (uint32_t)bits, (uint32_t)(bits >> 32));
    const uint32_t nruns = h.w >> 16;
    uint2 rr[kDescRuns];
#pragma unroll
    for (uint32_t k = 0; k < kDescRuns; k++) rr[k] = k < nruns ? q.p_runs[h.y + k] : make_uint2(0, 0);
#pragma unroll
    for (uint32_t k = 0; k < kDescRuns; k += 2)
      d[2 + k / 2] = make_uint4(rr[k].x, rr[k].y, rr[k + 1].x, rr[k + 1].y);
  }
  for (uint32_t k = threadIdx.x; k < q.p_nruns; k += blockDim.x) tile_runs[ro + k] = q.p_runs[k];
}

// What the producer hands the consumers with each ring stage (in shared
// memory beside the barriers, written before the stage's arrive).
struct MultiStageMeta {
  uint32_t model, r0, rows, w;
  unsigned long long bits;   // target rows of the tile
  unsigned long long first;  // lanes at their local step 1
  void *y;                   // the model's output buffer (vec[n & 1])
  long long *dots;           // the model's doubling sums
};
constexpr uint32_t kMultiHeader = 128 + kTiledMaxStages * 64;  // barriers, then a MultiStageMeta per stage
static_assert(sizeof(MultiStageMeta) <= 64, "a stage's meta takes one 64-byte slot");

// CV = 10*GA + PA splits the float -> FP64 widenings between the pipes as
// in kpm_step_tiled: the gathers of a row's first GA entries and, with PA,
// j_{n-1} widen on the integer pipe (f2d_scaled), the rest by conversion
// instructions on the XU pipe; every choice stores the same vectors.
template <bool CPLX, int TPR, int VPT, int R, int CW, int BPS, int CV>
__global__ void __launch_bounds__(32 * (CW + 1), BPS)
kpm_multi_tiled(const MultiModel *__restrict__ models, const MultiHeader *__restrict__ hdr,
                TiledLayout LY, uint32_t step_offset, uint32_t W, uint32_t ld, int *err,
                uint32_t wait_limit) {
  using E = typename TiledTypes<CPLX>::E;
  using Val = typename TiledTypes<CPLX>::Val;
  using Pk = typename std::conditional<CPLX, Pack<float2, TPR, VPT>, RPack<TPR, VPT>>::type;
  using L = typename Pk::L;
  constexpr int NL = Pk::NL;
  constexpr int GA = CV / 10;
  constexpr bool PA = CV % 10 != 0;
  constexpr int RPP = CW * 32 / TPR;  // rows per pass
  constexpr int PASSES = (R + RPP - 1) / RPP;
  static_assert(CW * 32 % TPR == 0, "a row group must divide the consumer threads");
  static_assert(R <= 64 && 64 % R == 0, "a tile's target bits are one 64-bit word");
  extern __shared__ __align__(128) unsigned char tsm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(tsm);
  uint64_t *empty = full + kTiledMaxStages;
  MultiStageMeta *smeta = reinterpret_cast<MultiStageMeta *>(tsm + 128);
  unsigned char *ring = tsm + kMultiHeader;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned fullmask = 0xffffffffu;
  const uint32_t S = LY.stages;
  const uint32_t rowbytes = W * (uint32_t)sizeof(E);
  const uint32_t total = hdr->total_tiles, run = hdr->run;
  const uint4 *__restrict__ tdesc = hdr->tile_desc;
  const uint2 *__restrict__ truns = hdr->tile_runs;
  const int32_t n = multi_step_index(hdr, step_offset);
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], CW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // the block's i-th tile: runs of `run` consecutive tiles, run b, b + grid, ...
  auto tile_at = [&](uint32_t i) -> uint32_t {
    return (blockIdx.x + (i / run) * gridDim.x) * run + i % run;
  };

  if (warp == 0) {
    // ---------------------------------------------------------- producer
    // Lane l < 12 holds 8 bytes of a tile's descriptor (lanes 0-1 the
    // header, 2-3 the meta word, 4-11 runs 0-7), loaded two tiles ahead, so
    // a tile's copies are issued without waiting on a load; a model's
    // pointers and first-step lanes are loaded when the model changes.
    auto load_desc = [&](uint32_t t) -> uint2 {
      return (t < total && lane < 12)
                 ? __ldg(reinterpret_cast<const uint2 *>(tdesc + (size_t)t * kDescWords) + lane)
                 : make_uint2(0, 0);
    };
    uint32_t t0 = tile_at(0), t1 = tile_at(1);
    uint2 d0 = load_desc(t0), d1 = load_desc(t1);
    uint32_t cq = kPad;
    const Val *m_val = nullptr;
    const uint16_t *m_slot = nullptr;
    const E *m_x = nullptr;
    E *m_y = nullptr;
    long long *m_dots = nullptr;
    unsigned long long m_first = 0;
    bool failed = false;
    uint32_t issued = 0;
    for (uint32_t i = 0; t0 < total; i++) {
      const uint32_t t2 = tile_at(i + 2);
      const uint2 d2 = load_desc(t2);
      const uint32_t h_ent = __shfl_sync(fullmask, d0.x, 0), h_run = __shfl_sync(fullmask, d0.y, 0);
      const uint32_t nuniq = __shfl_sync(fullmask, d0.x, 1), hw = __shfl_sync(fullmask, d0.y, 1);
      const uint32_t g_x = __shfl_sync(fullmask, d0.x, 2), r0 = __shfl_sync(fullmask, d0.y, 2);
      const uint32_t b_lo = __shfl_sync(fullmask, d0.x, 3), b_hi = __shfl_sync(fullmask, d0.y, 3);
      uint2 myrun;
      myrun.x = __shfl_sync(fullmask, d0.x, (lane + 4) & 31);
      myrun.y = __shfl_sync(fullmask, d0.y, (lane + 4) & 31);
      const uint32_t q0 = g_x & 0xffffu, Rt = g_x >> 16;
      if (q0 != cq) {
        cq = q0;
        const MultiModel *md = models + q0;
        m_val = static_cast<const Val *>(md->p_val);
        m_slot = md->p_slot;
        m_x = reinterpret_cast<const E *>(md->vec[(n + 1) & 1]);
        m_y = reinterpret_cast<E *>(md->vec[n & 1]);
        m_dots = md->dots;
        const int32_t *bs = md->base;
        const bool f0 = (uint32_t)lane < W && n - __ldg(bs + lane) == 1;
        const bool f1 = (uint32_t)lane + 32 < W && n - __ldg(bs + lane + 32) == 1;
        m_first = (unsigned long long)__ballot_sync(fullmask, f0) |
                  ((unsigned long long)__ballot_sync(fullmask, f1) << 32);
      }
      const uint32_t s = i % S;
      if (i >= S && !mbar_wait_limit(&empty[s], ((i / S) - 1) & 1u, wait_limit)) {
        failed = true;
        break;
      }
      unsigned char *st = ring + (size_t)s * LY.stage_bytes;
      const uint32_t w = hw & 0xffffu, nruns = hw >> 16;
      const uint32_t ebytes = w * R * (uint32_t)sizeof(Val), sbytes = w * R * 2u;
      const uint32_t bytes = (w ? ebytes + sbytes : 0u) + (2 * Rt + nuniq) * rowbytes;
      if (lane == 0) {
        MultiStageMeta &mt = smeta[s];
        mt.model = q0;
        mt.r0 = r0;
        mt.rows = Rt;
        mt.w = w;
        mt.bits = (unsigned long long)b_lo | ((unsigned long long)b_hi << 32);
        mt.first = m_first;
        mt.y = m_y;
        mt.dots = m_dots;
        // the arrive (release) orders the meta before the consumers' wait
        mbar_expect_tx(&full[s], bytes);
      }
      __syncwarp();
      const uint64_t e0 = (uint64_t)h_ent * R;
      if (w) {
        if (lane == 0) bulk_load(st, m_val + e0, ebytes, &full[s]);
        if (lane == 1) bulk_load(st + LY.off_slots, m_slot + e0, sbytes, &full[s]);
      }
      if (lane == 2) bulk_load(st + LY.off_xs, m_x + (uint64_t)r0 * W, Rt * rowbytes, &full[s]);
      if (lane == 3) bulk_load(st + LY.off_prev, m_y + (uint64_t)r0 * W, Rt * rowbytes, &full[s]);
      for (uint32_t c = 0; c < nruns; c += 32) {
        uint2 rn = myrun;
        if (c > 0 || lane >= (int)kDescRuns)
          rn = (c + lane < nruns) ? __ldg(truns + h_run + c + lane) : make_uint2(0, 0);
        if (c + lane < nruns) {
          const uint32_t slot = R + (rn.y >> 16), len = rn.y & 0xffffu;
          bulk_load(st + LY.off_xs + (size_t)slot * rowbytes, m_x + (uint64_t)rn.x * W,
                    len * rowbytes, &full[s]);
        }
      }
      issued = i + 1;
      t0 = t1;
      d0 = d1;
      t1 = t2;
      d1 = d2;
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
    // Everything a tile needs besides its staged rows comes with the stage
    // (MultiStageMeta); only target rows read the model's target list.
    const int ct = threadIdx.x - 32;
    const int sub = ct % TPR, grp = ct / TPR;
    uint32_t cq = kPad;
    long long *t_dots = nullptr;
    E *m_y = nullptr;
    uint32_t first = 0;
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
          a += __shfl_xor_sync(fullmask, a, off);
          b += __shfl_xor_sync(fullmask, b, off);
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
    for (uint32_t i = 0; tile_at(i) < total; i++) {
      const uint32_t s = i % S;
      if (!mbar_wait_limit(&full[s], (i / S) & 1u, wait_limit)) {
        failed = true;
        break;
      }
      const MultiStageMeta mt = smeta[s];
      if (mt.model != cq) {
        if (cq != kPad) flush();
        cq = mt.model;
        t_dots = mt.dots;
        m_y = static_cast<E *>(mt.y);
        first = 0;
#pragma unroll
        for (int j = 0; j < VPT; j++)
          if ((mt.first >> Pk::col_of(sub, j)) & 1ull) first |= 1u << j;
      }
      const uint32_t w = mt.w, r0 = mt.r0, Rt = mt.rows;
      const unsigned long long bits = mt.bits;
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
        // moments of this row's targets (rare: the rows of lane sources and
        // Green's-function to-indices)
        auto targets = [&](auto store) {
          const MultiModel *md = models + cq;
          const uint32_t *t_row = md->trow, *t_col = md->tcol;
          const uint32_t t_count = md->tcount;
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
            double2 *dst = multi_target_dst(md, tc, n - __ldg(md->base + c), ld);
            if (dst) store(dst, jt);
          }
        };
        if constexpr (CPLX) {
          double2 acc[VPT];
          {
            L yv[NL];
            Pk::load_rw(reinterpret_cast<const float2 *>(prev) + (size_t)lr * W, sub, yv);
#pragma unroll
            for (int j = 0; j < VPT; j++) {
              double2 f;
              if constexpr (PA) {
                const float2 g = Pk::getf(yv, j);
                f = make_double2(f2d_scaled(g.x) * kWideUp, f2d_scaled(g.y) * kWideUp);
              } else {
                f = Pk::get(yv, j);
              }
              acc[j] = ((first >> j) & 1u) ? make_double2(0.0, 0.0) : make_double2(-f.x, -f.y);
            }
          }
          for (uint32_t k = 0; k < w; k++) {
            const uint16_t sl = slots[k * R + lr];
            if (sl == kSlotPad) break;
            const double2 v = vals[k * R + lr];
            L xr[NL];
            Pk::load_rw(reinterpret_cast<const float2 *>(xs) + (size_t)sl * W, sub, xr);
            if (GA > 0 && k < (uint32_t)GA) {
              const double2 vu = make_double2(v.x * kWideUp, v.y * kWideUp);
#pragma unroll
              for (int j = 0; j < VPT; j++) {
                const float2 f = Pk::getf(xr, j);
                acc[j] = cmac<false>(acc[j], vu, make_double2(f2d_scaled(f.x), f2d_scaled(f.y)));
              }
            } else {
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[j] = cmac<false>(acc[j], v, Pk::get(xr, j));
            }
          }
#pragma unroll
          for (int j = 0; j < VPT; j++)
            if ((first >> j) & 1u) acc[j] = make_double2(acc[j].x * 0.5, acc[j].y * 0.5);
          if ((bits >> lr) & 1ull)
            targets([&](double2 *dst, int jt) {
#pragma unroll
              for (int j = 0; j < VPT; j++)
                if (j == jt) *dst = acc[j];
            });
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
            for (int j = 0; j < VPT; j++) {
              const float f = Pk::getf(yv, j);
              acc[j] = ((first >> j) & 1u) ? 0.0 : (PA ? f2d_scaled(f) * -kWideUp : -(double)f);
            }
          }
          for (uint32_t k = 0; k < w; k++) {
            const uint16_t sl = slots[k * R + lr];
            if (sl == kSlotPad) break;
            const double v = vals[k * R + lr];
            L xr[NL];
            Pk::load_rw(reinterpret_cast<const float *>(xs) + (size_t)sl * W, sub, xr);
            if (GA > 0 && k < (uint32_t)GA) {
              const double vu = v * kWideUp;
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[j] = fma(vu, f2d_scaled(Pk::getf(xr, j)), acc[j]);
            } else {
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[j] = fma(v, (double)Pk::getf(xr, j), acc[j]);
            }
          }
#pragma unroll
          for (int j = 0; j < VPT; j++)
            if ((first >> j) & 1u) acc[j] = acc[j] * 0.5;
          if ((bits >> lr) & 1ull)
            targets([&](double2 *dst, int jt) {
#pragma unroll
              for (int j = 0; j < VPT; j++)
                if (j == jt) *dst = make_double2(acc[j], 0.0);
            });
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
template <bool CPLX, int TPR, int VPT, int R, int CW, int BPS, int CV>
void launch_multi_tiled(cudaStream_t st, int device, const MultiModel *models,
                        const MultiHeader *hdr, uint32_t step_offset, uint32_t W, uint32_t ld,
                        const MultiLaunch &ml) {
  auto kern = kpm_multi_tiled<CPLX, TPR, VPT, R, CW, BPS, CV>;
  if (ml.ly.stages == 0) return;
  static bool attr[64] = {false};
  const int d = device & 63;
  if (!attr[d]) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tiled_budget(BPS));
    attr[d] = true;
  }
  const uint32_t smem = kMultiHeader + ml.ly.stages * ml.ly.stage_bytes;
  kern<<<(unsigned)(BPS * sm_count(device)), 32 * (CW + 1), smem, st>>>(
      models, hdr, ml.ly, step_offset, W, ld, ml.err, ml.wait_limit);
}

#define TBTKKPM_MULTI_TILED_ENTRY(CPLX, T, P, R, CW, BPS, CV)                          \
  {T, P, kMultiTiledVariant + 1000000 * CV + 1000 * R + 10 * CW + BPS,                  \
   &launch_multi_tiled<CPLX, T, P, R, CW, BPS, CV>}

extern const MultiEntry kMultiTiled[];
extern const int kNumMultiTiled;
extern const MultiEntry kMultiTiledReal[];
extern const int kNumMultiTiledReal;

}  // namespace tbtkkpm
