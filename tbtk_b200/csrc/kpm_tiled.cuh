// Tile-staged recursion step: the gathered rows of a tile of R consecutive
// output rows are staged in shared memory by bulk asynchronous copies, one
// copy per run of consecutive columns.
//
// Why: a tight-binding row gathers j_n at a handful of columns, and the rows
// of a tile of consecutive rows gather mostly the same columns (a lattice
// site's neighbours are its tile-mates or a lattice row up or down).  The
// matrix builder (k_plan_count / k_plan_fill below) lists, per tile, the
// distinct columns outside the tile, sorted and merged into runs of
// consecutive columns; on the 2048^2 spin lattice a 64-row tile has about
// 132 such columns in 3-4 runs.  The step then moves each distinct row of
// j_n once into shared memory (own rows + runs), so
// * the bytes in flight per SM are set by the shared-memory ring (up to
//   227 KB), not by registers: a producer warp issues the copies of whole
//   tiles ahead while 4-16 consumer warps compute from shared memory;
// * a lattice row costs a few 16-64 KB copies instead of one dependent
//   load per entry, so the step is not bound by memory latency;
// * the row's own j_n, which the doubling dot products need, is already in
//   shared memory (the tile's own rows are always staged first).
//
// The plan of a tile: a header {ent_begin, run_begin, nuniq, w | nruns<<16},
// its runs {first column, slot_start << 16 | length}, and its entries in
// [w][R] layout: the shared-memory slot of each entry's column (own rows at
// slots 0..R-1, run rows from slot R on; 0xffff in padding) and its value
// 2H/s.  Entries keep the CSR order of their row (ascending columns), so each
// element sees the same FMAs in the same order as kpm_step_real /
// kpm_step<float2, Wide64>: stored vectors and directly gathered moments are
// bit-identical to theirs.  The FP64 form stages complex128 rows and keeps
// the reference's rounded products and sums (as kpm_step<double2, Exact64>).
//
// Only non-multicast bulk copies are issued.  Every mbarrier wait is
// bounded (`wait_limit` polls; 0 gives up at once); a wait that runs out
// sets *err and ends the loops, and before the block exits every copy it
// issued has landed (waited for with the library's bound kWaitLimit).
#pragma once

#include "kpm_bulk.cuh"
#include "kpm_host.h"
#include "kpm_real.cuh"

namespace tbtkkpm {

constexpr uint16_t kSlotPad = 0xffff;
// a row-pair plan entry: bits 0-13 the slot, bit 14 the pair's first row
// has the column, bit 15 its second row (kSlotPad: padding)
constexpr uint32_t kPairSlotBits = 0x3fffu;
constexpr uint32_t kPlanCap = 4096;  // entries of one tile the plan builder sorts
constexpr int kPlanBlock = 256;
constexpr uint32_t kTiledMaxStages = 8;
constexpr uint32_t kTiledHeader = 256;  // barriers at the start of dynamic shared memory

__host__ __device__ inline uint32_t align_up(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

// Shared memory a tile-staged block may use with BPS blocks per SM (the SM
// has 228 KB; each block reserves 1 KB; one block may take at most 227 KB).
constexpr uint32_t tiled_budget(int bps) {
  return bps <= 1 ? 232448u : 233472u / (uint32_t)bps - 1024u;
}

// Layout of a stage for `rowbytes` bytes per vector row and `vbytes` per
// value; stages = 0 when fewer than two stages fit `budget` bytes.
inline TiledLayout tiled_layout(const TilePlan &p, uint32_t rowbytes, uint32_t vbytes,
                                uint32_t budget) {
  TiledLayout L{};
  L.off_slots = align_up(p.wmax * p.R * vbytes, 128);
  L.off_xs = L.off_slots + align_up(p.wmax * p.R * 2, 128);
  L.off_prev = L.off_xs + (p.R + p.umax) * rowbytes;
  L.stage_bytes = align_up(L.off_prev + p.R * rowbytes, 128);
  const uint32_t usable = budget > kTiledHeader ? budget - kTiledHeader : 0;
  uint32_t s = L.stage_bytes ? usable / L.stage_bytes : 0;
  if (s > kTiledMaxStages) s = kTiledMaxStages;
  L.stages = s >= 2 ? s : 0;
  return L;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_wait_limit(uint64_t *bar, uint32_t parity, uint32_t limit) {
  for (uint32_t it = 0; it < limit; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Widening of a float to FP64 on the integer pipe: the float's exponent and
// mantissa fields moved into the double's fields (shift right by 3, sign
// kept by the arithmetic shift and a mask; the low 3 mantissa bits into the
// low word) read the float's exponent bias 127 as the double's 1023, so the
// double is x * 2^-896 exactly, for normal and subnormal floats alike (a
// float subnormal becomes the double subnormal of the same scaled value),
// and zero stays zero.  Infinite and NaN floats do not occur (finite matrix
// values, |j_n| <= 1).  The recursion multiplies such a value by the entry
// value scaled up by 2^896 (exact): the FMA's exact product equals v * x,
// so the rounded result is the same as with a conversion instruction,
// which runs on the 16-per-clock XU pipe.
__device__ __forceinline__ double f2d_scaled(float x) {
  const int b = __float_as_int(x);
  return __hiloint2double((b >> 3) & (int)0x8fffffff, b << 29);
}
constexpr double kWideUp = 0x1p896;

// Element type of a vector row and value type of an entry (F64: the
// complex128 vectors of the FP64 recursion).
template <bool CPLX, bool F64 = false> struct TiledTypes;
template <> struct TiledTypes<false, false> {
  using E = float;
  using Val = double;
};
template <> struct TiledTypes<true, false> {
  using E = float2;
  using Val = double2;
};
template <> struct TiledTypes<true, true> {
  using E = double2;
  using Val = double2;
};

// One recursion step over the tiles of `P` (same outputs as kpm_step_real
// for CPLX false, kpm_step<float2, Wide64> for CPLX true).  Warp 0 is the
// producer; warps 1..CW consume.  Consumer thread `sub` of a TPR-thread
// group owns VPT elements of its row (interleaved 16-byte chunks, as
// RPack / Pack), and the CW*32/TPR groups take the tile's rows in passes.
// CV = 100*PAIR + 10*GA + PA.  GA and PA split the float -> FP64 widenings
// between the pipes: the gathers of a row's first GA entries and, with PA,
// j_{n-1} and the dot-product terms widen on the integer pipe
// (f2d_scaled), the rest by conversion instructions.  PAIR (complex
// vectors, R >= 16) reads a row-pair plan (tile_plan with pairs): a group
// takes two adjacent rows, walks the merge of their column lists and
// widens each gathered row once for both (a spin lattice site's two rows
// share most columns), adding it into each row that has the column; each
// row still sees its own entries in CSR order.  Every choice gives the same
// stored vectors.
//
// F64 (complex, CV 0, no dot products): the FP64 recursion on complex128
// vectors in the reference's operation order (Exact64: each row's sum starts
// at -j_{n-1} and adds every complex product, each rounded once, in CSR
// order, Lib/src/Solver/ChebyshevExpander.cpp:171-186), the same as
// kpm_step<double2, Exact64>: moments bit-identical to the reference's.
template <bool CPLX, int TPR, int VPT, int R, int CW, int BPS, bool FIRST, bool DOTS, int CV = 0,
          bool F64 = false>
__global__ void __launch_bounds__(32 * (CW + 1), BPS)
kpm_step_tiled(TilePlan P, TiledLayout LY, uint32_t Bp,
               const typename TiledTypes<CPLX, F64>::E *__restrict__ x,
               typename TiledTypes<CPLX, F64>::E *__restrict__ y, Targets tg, uint32_t n_out,
               double2 *__restrict__ dots, int *err, uint32_t wait_limit) {
  using E = typename TiledTypes<CPLX, F64>::E;
  using Val = typename TiledTypes<CPLX, F64>::Val;
  using Pk = typename std::conditional<
      CPLX, typename std::conditional<F64, Pack<double2, TPR, VPT>, Pack<float2, TPR, VPT>>::type,
      RPack<TPR, VPT>>::type;
  using L = typename Pk::L;
  constexpr int NL = Pk::NL;
  constexpr bool PAIR = CV >= 100;
  constexpr int GA = (CV % 100) / 10;
  constexpr bool PA = CV % 10 != 0;
  constexpr int RPP = CW * 32 / TPR;  // row units (rows, or row pairs) per pass
  constexpr uint32_t EW = PAIR ? R / 2 : R;  // plan entries of one chunk row: a row or a pair
  constexpr int PASSES = ((int)EW + RPP - 1) / RPP;
  static_assert(CW * 32 % TPR == 0, "a row group must divide the consumer threads");
  static_assert(!PAIR || (CPLX && R >= 16), "row pairs: complex vectors, 16-byte slot chunks");
  static_assert(!F64 || (CPLX && CV == 0 && !DOTS), "FP64 steps: complex values, every moment direct");
  extern __shared__ __align__(128) unsigned char tsm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(tsm);
  uint64_t *empty = full + kTiledMaxStages;
  unsigned char *ring = tsm + kTiledHeader;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t S = LY.stages;
  const uint32_t rowbytes = Bp * (uint32_t)sizeof(E);
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], CW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const int ct = threadIdx.x - 32;
  const int sub = ct >= 0 ? ct % TPR : 0, grp = ct >= 0 ? ct / TPR : 0;
  double d_nn[DOTS ? VPT : 1], d_np[DOTS ? VPT : 1];
#pragma unroll
  for (int j = 0; j < (DOTS ? VPT : 1); j++) d_nn[j] = d_np[j] = 0.0;

  if (warp == 0) {
    // ---------------------------------------------------------- producer
    // Headers two tiles ahead and the first 32 runs one tile ahead, so the
    // header -> runs -> copies chain is off the issue path.
    const uint32_t G = gridDim.x;
    uint32_t t = blockIdx.x;
    uint4 h0 = make_uint4(0, 0, 0, 0), h1 = h0;
    if (t < P.ntiles) h0 = __ldg(P.hdr + t);
    if (t + G < P.ntiles) h1 = __ldg(P.hdr + t + G);
    uint2 run0 = make_uint2(0, 0);
    if (t < P.ntiles && (uint32_t)lane < (h0.w >> 16)) run0 = __ldg(P.runs + h0.y + lane);
    bool failed = false;
    uint32_t issued = 0;  // tiles whose copies were issued (tile i into stage i % S)
    for (uint32_t i = 0; t < P.ntiles; t += G, i++) {
      uint4 h2 = make_uint4(0, 0, 0, 0);
      if (t + 2 * G < P.ntiles) h2 = __ldg(P.hdr + t + 2 * G);
      uint2 run1 = make_uint2(0, 0);
      if (t + G < P.ntiles && (uint32_t)lane < (h1.w >> 16)) run1 = __ldg(P.runs + h1.y + lane);
      const uint32_t s = i % S;
      if (i >= S && !mbar_wait_limit(&empty[s], ((i / S) - 1) & 1u, wait_limit)) {
        failed = true;
        break;
      }
      unsigned char *st = ring + (size_t)s * LY.stage_bytes;
      const uint32_t w = h0.w & 0xffffu, nruns = h0.w >> 16, nuniq = h0.z;
      const uint32_t r0 = t * R, Rt = min((uint32_t)R, P.N - r0);
      // pair entries carry two values each: w * R values either way
      const uint32_t ebytes = w * R * (uint32_t)sizeof(Val), sbytes = w * EW * 2u;
      const uint32_t bytes =
          ebytes + sbytes + (Rt + nuniq + (FIRST ? 0u : Rt)) * rowbytes;
      if (lane == 0) mbar_expect_tx(&full[s], bytes);
      __syncwarp();
      const uint64_t e0 = (uint64_t)h0.x * EW;
      if (w) {
        if (lane == 0)
          bulk_load(st, static_cast<const Val *>(P.eval) + e0 * (PAIR ? 2 : 1), ebytes, &full[s]);
        if (lane == 1) bulk_load(st + LY.off_slots, P.eslot + e0, sbytes, &full[s]);
      }
      if (lane == 2) bulk_load(st + LY.off_xs, x + (uint64_t)r0 * Bp, Rt * rowbytes, &full[s]);
      if (!FIRST && lane == 3)
        bulk_load(st + LY.off_prev, y + (uint64_t)r0 * Bp, Rt * rowbytes, &full[s]);
      for (uint32_t c = 0; c < nruns; c += 32) {
        uint2 rn = run0;
        if (c > 0) rn = (c + lane < nruns) ? __ldg(P.runs + h0.y + c + lane) : make_uint2(0, 0);
        if (c + lane < nruns) {
          const uint32_t slot = R + (rn.y >> 16), len = rn.y & 0xffffu;
          bulk_load(st + LY.off_xs + (size_t)slot * rowbytes, x + (uint64_t)rn.x * Bp,
                    len * rowbytes, &full[s]);
        }
      }
      issued = i + 1;
      h0 = h1;
      h1 = h2;
      run0 = run1;
    }
    if (failed && lane == 0) atomicExch(err, kErrTimeout);
    // every copy issued into this block's ring has landed (or its wait ran
    // out) before the ring is reused or the block exits; this wait keeps the
    // library's bound whatever `wait_limit` the step was given
    if (lane == 0)
      for (uint32_t s = 0; s < S && s < issued; s++) {
        const uint32_t fills = (issued - 1 - s) / S + 1;
        if (!mbar_wait_limit(&full[s], (fills - 1) & 1u, kWaitLimit)) atomicExch(err, kErrTimeout);
      }
  } else {
    // ---------------------------------------------------------- consumers
    bool failed = false;
    for (uint32_t i = 0, t = blockIdx.x; t < P.ntiles; t += gridDim.x, i++) {
      const uint32_t s = i % S;
      const uint4 h = __ldg(P.hdr + t);
      const uint32_t w = h.w & 0xffffu;
      const uint32_t r0 = t * R, Rt = min((uint32_t)R, P.N - r0);
      uint32_t bw[PASSES];
#pragma unroll
      for (int p = 0; p < PASSES; p++) {
        const uint32_t lr = (grp + p * RPP) * (PAIR ? 2 : 1);  // a pair's rows share a word
        bw[p] = lr < Rt ? __ldg(tg.bitmap + ((r0 + lr) >> 5)) : 0u;
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
        if constexpr (F64) {
          const uint32_t lr = grp + p * RPP;
          if (lr >= Rt) continue;
          const uint32_t row = r0 + lr;
          double2 acc[VPT];
          if constexpr (FIRST) {
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = make_double2(0.0, 0.0);
          } else {
            L yv[NL];
            Pk::load_rw(reinterpret_cast<const double2 *>(prev) + (size_t)lr * Bp, sub, yv);
#pragma unroll
            for (int j = 0; j < VPT; j++) {
              const double2 f = Pk::get(yv, j);
              acc[j] = make_double2(-f.x, -f.y);
            }
          }
          for (uint32_t k = 0; k < w; k++) {
            const uint16_t sl = slots[k * R + lr];
            if (sl == kSlotPad) break;
            double2 v = vals[k * R + lr];
            if constexpr (FIRST) v = make_double2(v.x * 0.5, v.y * 0.5);
            L xr[NL];
            Pk::load_rw(reinterpret_cast<const double2 *>(xs) + (size_t)sl * Bp, sub, xr);
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = cmac<true>(acc[j], v, Pk::get(xr, j));
          }
          if ((bw[p] >> (row & 31)) & 1u) {
            for (uint32_t q = target_first(tg, row); q < tg.count && __ldg(tg.row + q) == row; q++) {
              const int jt = Pk::slot_of(sub, __ldg(tg.col + q));
              if (jt >= 0) {
#pragma unroll
                for (int j = 0; j < VPT; j++)
                  if (j == jt) tg.mu[(uint64_t)__ldg(tg.out + q) * tg.ld + n_out] = acc[j];
              }
            }
          }
          Pk::store(reinterpret_cast<double2 *>(y) + (uint64_t)row * Bp, sub, acc);
          continue;
        }
        if constexpr (PAIR) {
          const uint32_t u = grp + p * RPP, la = 2 * u;
          if (la >= Rt) continue;
          const bool hb = la + 1 < Rt;
          double2 acc[2][VPT];
#pragma unroll
          for (int h = 0; h < 2; h++) {
            if (FIRST || (h == 1 && !hb)) {
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[h][j] = make_double2(0.0, 0.0);
            } else {
              L yv[NL];
              Pk::load_rw(reinterpret_cast<const float2 *>(prev) + (size_t)(la + h) * Bp, sub, yv);
#pragma unroll
              for (int j = 0; j < VPT; j++) {
                const float2 f = Pk::getf(yv, j);
                if constexpr (PA)
                  acc[h][j] = make_double2(f2d_scaled(f.x) * -kWideUp, f2d_scaled(f.y) * -kWideUp);
                else
                  acc[h][j] = make_double2(-(double)f.x, -(double)f.y);
              }
            }
          }
          for (uint32_t k = 0; k < w; k++) {
            const uint16_t sl = slots[k * EW + u];
            if (sl == kSlotPad) break;
            const uint32_t mask = sl >> 14, slot = sl & kPairSlotBits;
            double2 va = vals[2 * (k * EW + u)], vb = vals[2 * (k * EW + u) + 1];
            if constexpr (FIRST) {
              va = make_double2(va.x * 0.5, va.y * 0.5);
              vb = make_double2(vb.x * 0.5, vb.y * 0.5);
            }
            L xr[NL];
            Pk::load_rw(reinterpret_cast<const float2 *>(xs) + (size_t)slot * Bp, sub, xr);
            const bool scaled = GA > 0 && k < (uint32_t)GA;
            if (scaled) {
              va = make_double2(va.x * kWideUp, va.y * kWideUp);
              vb = make_double2(vb.x * kWideUp, vb.y * kWideUp);
            }
            double2 xd[VPT];
#pragma unroll
            for (int j = 0; j < VPT; j++) {
              const float2 f = Pk::getf(xr, j);
              xd[j] = scaled ? make_double2(f2d_scaled(f.x), f2d_scaled(f.y))
                             : make_double2((double)f.x, (double)f.y);
            }
            if (mask & 1u) {
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[0][j] = cmac<false>(acc[0][j], va, xd[j]);
            }
            if (mask & 2u) {
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[1][j] = cmac<false>(acc[1][j], vb, xd[j]);
            }
          }
#pragma unroll
          for (int h = 0; h < 2; h++) {
            if (h == 1 && !hb) break;
            const uint32_t lr = la + h, row = r0 + lr;
            if ((bw[p] >> (row & 31)) & 1u) {
              for (uint32_t q = target_first(tg, row); q < tg.count && __ldg(tg.row + q) == row; q++) {
                const int jt = Pk::slot_of(sub, __ldg(tg.col + q));
                if (jt >= 0) {
#pragma unroll
                  for (int j = 0; j < VPT; j++)
                    if (j == jt) tg.mu[(uint64_t)__ldg(tg.out + q) * tg.ld + n_out] = acc[h][j];
                }
              }
            }
            float2 af[VPT];
#pragma unroll
            for (int j = 0; j < VPT; j++)
              af[j] = make_float2(__double2float_rn(acc[h][j].x), __double2float_rn(acc[h][j].y));
            Pk::storef(reinterpret_cast<float2 *>(y) + (uint64_t)row * Bp, sub, af);
            if constexpr (DOTS) {
              L self[NL];
              Pk::load_rw(reinterpret_cast<const float2 *>(xs) + (size_t)lr * Bp, sub, self);
#pragma unroll
              for (int j = 0; j < VPT; j++) {
                const float2 b = Pk::getf(self, j);
                const float nn = fmaf(af[j].x, af[j].x, af[j].y * af[j].y);
                const float np = fmaf(af[j].x, b.x, af[j].y * b.y);
                d_nn[j] += PA ? f2d_scaled(nn) : (double)nn;
                d_np[j] += PA ? f2d_scaled(np) : (double)np;
              }
            }
          }
          continue;
        }
        const uint32_t lr = grp + p * RPP;
        if (lr >= Rt) continue;
        const uint32_t row = r0 + lr;
        if constexpr (CPLX && !F64) {
          double2 acc[VPT];
          if constexpr (FIRST) {
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = make_double2(0.0, 0.0);
          } else {
            L yv[NL];
            Pk::load_rw(reinterpret_cast<const float2 *>(prev) + (size_t)lr * Bp, sub, yv);
#pragma unroll
            for (int j = 0; j < VPT; j++) {
              const float2 f = Pk::getf(yv, j);
              if constexpr (PA)
                acc[j] = make_double2(f2d_scaled(f.x) * -kWideUp, f2d_scaled(f.y) * -kWideUp);
              else
                acc[j] = make_double2(-(double)f.x, -(double)f.y);
            }
          }
          for (uint32_t k = 0; k < w; k++) {
            const uint16_t sl = slots[k * R + lr];
            if (sl == kSlotPad) break;
            double2 v = vals[k * R + lr];
            if constexpr (FIRST) v = make_double2(v.x * 0.5, v.y * 0.5);
            L xr[NL];
            Pk::load_rw(reinterpret_cast<const float2 *>(xs) + (size_t)sl * Bp, sub, xr);
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
          if ((bw[p] >> (row & 31)) & 1u) {
            for (uint32_t q = target_first(tg, row); q < tg.count && __ldg(tg.row + q) == row; q++) {
              const int jt = Pk::slot_of(sub, __ldg(tg.col + q));
              if (jt >= 0) {
#pragma unroll
                for (int j = 0; j < VPT; j++)
                  if (j == jt) tg.mu[(uint64_t)__ldg(tg.out + q) * tg.ld + n_out] = acc[j];
              }
            }
          }
          float2 af[VPT];
#pragma unroll
          for (int j = 0; j < VPT; j++)
            af[j] = make_float2(__double2float_rn(acc[j].x), __double2float_rn(acc[j].y));
          Pk::storef(reinterpret_cast<float2 *>(y) + (uint64_t)row * Bp, sub, af);
          if constexpr (DOTS) {
            L self[NL];
            Pk::load_rw(reinterpret_cast<const float2 *>(xs) + (size_t)lr * Bp, sub, self);
#pragma unroll
            for (int j = 0; j < VPT; j++) {
              const float2 b = Pk::getf(self, j);
              const float nn = fmaf(af[j].x, af[j].x, af[j].y * af[j].y);
              const float np = fmaf(af[j].x, b.x, af[j].y * b.y);
              d_nn[j] += PA ? f2d_scaled(nn) : (double)nn;
              d_np[j] += PA ? f2d_scaled(np) : (double)np;
            }
          }
        } else if constexpr (!CPLX) {
          double acc[VPT];
          if constexpr (FIRST) {
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = 0.0;
          } else {
            L yv[NL];
            Pk::load_rw(reinterpret_cast<const float *>(prev) + (size_t)lr * Bp, sub, yv);
#pragma unroll
            for (int j = 0; j < VPT; j++) {
              const float f = Pk::getf(yv, j);
              acc[j] = PA ? f2d_scaled(f) * -kWideUp : -(double)f;
            }
          }
          for (uint32_t k = 0; k < w; k++) {
            const uint16_t sl = slots[k * R + lr];
            if (sl == kSlotPad) break;
            double v = vals[k * R + lr];
            if constexpr (FIRST) v = v * 0.5;
            L xr[NL];
            Pk::load_rw(reinterpret_cast<const float *>(xs) + (size_t)sl * Bp, sub, xr);
            if (GA > 0 && k < (uint32_t)GA) {
              const double vu = v * kWideUp;
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[j] = fma(vu, f2d_scaled(Pk::getf(xr, j)), acc[j]);
            } else {
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[j] = fma(v, (double)Pk::getf(xr, j), acc[j]);
            }
          }
          if ((bw[p] >> (row & 31)) & 1u) {
            for (uint32_t q = target_first(tg, row); q < tg.count && __ldg(tg.row + q) == row; q++) {
              const int jt = Pk::slot_of(sub, __ldg(tg.col + q));
              if (jt >= 0) {
#pragma unroll
                for (int j = 0; j < VPT; j++)
                  if (j == jt)
                    tg.mu[(uint64_t)__ldg(tg.out + q) * tg.ld + n_out] = make_double2(acc[j], 0.0);
              }
            }
          }
          float af[VPT];
#pragma unroll
          for (int j = 0; j < VPT; j++) af[j] = __double2float_rn(acc[j]);
          Pk::storef(reinterpret_cast<float *>(y) + (uint64_t)row * Bp, sub, af);
          if constexpr (DOTS) {
            L self[NL];
            Pk::load_rw(reinterpret_cast<const float *>(xs) + (size_t)lr * Bp, sub, self);
#pragma unroll
            for (int j = 0; j < VPT; j++) {
              const float b = Pk::getf(self, j);
              const float nn = fmaf(af[j], af[j], 0.0f), np = fmaf(af[j], b, 0.0f);
              d_nn[j] += PA ? f2d_scaled(nn) : (double)nn;
              d_np[j] += PA ? f2d_scaled(np) : (double)np;
            }
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
    if (failed && lane == 0) atomicExch(err, kErrTimeout);
  }
  if constexpr (DOTS) {
    // per-thread sums, then a fixed-order sum over the block's row groups;
    // the ring is free (every issued copy has landed, see the producer)
    __syncthreads();
    double *red = reinterpret_cast<double *>(ring);  // [CW*32][2]
#pragma unroll
    for (int j = 0; j < VPT; j++) {
      if (ct >= 0) {
        // sums of terms widened on the integer pipe carry the 2^-896 scale
        red[2 * ct] = PA ? d_nn[j] * kWideUp : d_nn[j];
        red[2 * ct + 1] = PA ? d_np[j] * kWideUp : d_np[j];
      }
      __syncthreads();
      if (ct >= 0 && grp == 0) {
        double a = 0.0, b = 0.0;
        for (int r = 0; r < RPP; r++) {
          a += red[2 * (r * TPR + sub)];
          b += red[2 * (r * TPR + sub) + 1];
        }
        double2 *o = dots + (uint64_t)blockIdx.x * 2 * Bp;
        const uint32_t c = Pk::col_of(sub, j);
        o[c] = make_double2(a, 0.0);
        o[Bp + c] = make_double2(b, 0.0);
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------ plan builder
// One block of kPlanBlock threads per tile (grid-stride).  The tile's CSR
// entries are contiguous ([rowptr[r0], rowptr[r1])); their columns outside
// the tile are sorted in shared memory (bitonic), and the distinct ones and
// the runs of consecutive ones counted (k_plan_count) or listed
// (k_plan_fill).  A tile with more than kPlanCap entries sets *bad.

// Loads the tile's outside columns into keys[0, n2) (n2 = next power of two
// of the entry count, padded with kPad) and sorts them ascending.
__device__ inline uint32_t plan_sort_tile(uint32_t *keys, const uint32_t *col, uint32_t e0,
                                          uint32_t T, uint32_t r0, uint32_t r1) {
  uint32_t n2 = 1;
  while (n2 < T) n2 <<= 1;
  for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
    uint32_t k = kPad;
    if (i < T) {
      const uint32_t c = col[e0 + i];
      k = (c >= r0 && c < r1) ? kPad : c;
    }
    keys[i] = k;
  }
  __syncthreads();
  for (uint32_t size = 2; size <= n2; size <<= 1)
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
        const uint32_t j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const uint32_t a = keys[i], b = keys[j];
          if ((a > b) == up) {
            keys[i] = b;
            keys[j] = a;
          }
        }
      }
      __syncthreads();
    }
  return n2;
}

// flags of sorted position i: bit 0 a new distinct column, bit 1 the start
// of a run of consecutive columns
__device__ __forceinline__ uint32_t plan_flags(const uint32_t *keys, uint32_t i) {
  const uint32_t k = keys[i];
  if (k == kPad) return 0;
  if (i > 0 && keys[i - 1] == k) return 0;
  const bool run = i == 0 || keys[i - 1] != k - 1;
  return 1u | (run ? 2u : 0u);
}

// Exclusive block scan of v over the calling block (kPlanBlock threads);
// returns the prefix of this thread and the block total in *total.
__device__ inline uint32_t plan_block_scan(uint32_t v, uint32_t *total) {
  __shared__ uint32_t wsum[kPlanBlock / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  uint32_t before = 0, all = 0;
  for (int w = 0; w < kPlanBlock / 32; w++) {
    if (w < wid) before += wsum[w];
    all += wsum[w];
  }
  __syncthreads();
  *total = all;
  return before + inc - v;
}

template <int R>
__global__ void __launch_bounds__(kPlanBlock)
k_plan_count(uint32_t N, uint32_t ntiles, const uint32_t *__restrict__ rowptr,
             const uint32_t *__restrict__ col, uint32_t *tw, uint32_t *truns, uint32_t *tuniq,
             unsigned *maxes, unsigned *bad) {
  extern __shared__ uint32_t pkeys[];
  __shared__ unsigned cnt[3];
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t r0 = t * R, r1 = min(r0 + R, N);
    const uint32_t e0 = rowptr[r0], T = rowptr[r1] - e0;
    if (T > kPlanCap) {
      if (threadIdx.x == 0) {
        atomicOr(bad, 1u);
        tw[t] = truns[t] = tuniq[t] = 0;
      }
      continue;
    }
    if (threadIdx.x < 3) cnt[threadIdx.x] = 0;
    const uint32_t n2 = plan_sort_tile(pkeys, col, e0, T, r0, r1);
    uint32_t nu = 0, nr = 0, wmax = 0;
    for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
      const uint32_t f = plan_flags(pkeys, i);
      nu += f & 1u;
      nr += f >> 1;
    }
    for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x)
      wmax = max(wmax, rowptr[r + 1] - rowptr[r]);
    atomicAdd(&cnt[0], nu);
    atomicAdd(&cnt[1], nr);
    atomicMax(&cnt[2], wmax);
    __syncthreads();
    if (threadIdx.x == 0) {
      tuniq[t] = cnt[0];
      truns[t] = cnt[1];
      tw[t] = cnt[2];
      atomicMax(&maxes[0], cnt[0]);
      atomicMax(&maxes[1], cnt[2]);
    }
    __syncthreads();
  }
}

// Row-pair plans: the entries of a pair of rows (2u, 2u + 1 of a tile) are
// the merge of their ascending column lists, one entry per distinct column.
// tw[t] becomes the tile's most merged entries of a pair, maxes[3] the
// most of any tile (one thread per pair).
template <int R>
__global__ void __launch_bounds__(kPlanBlock)
k_plan_pair_width(uint32_t N, uint32_t ntiles, const uint32_t *__restrict__ rowptr,
                  const uint32_t *__restrict__ col, uint32_t *tw, unsigned *maxes) {
  const uint64_t pairs = (uint64_t)ntiles * (R / 2);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < pairs;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t t = (uint32_t)(i / (R / 2)), u = (uint32_t)(i % (R / 2));
    const uint32_t a = t * R + 2 * u, b = a + 1;
    uint32_t n = 0;
    if (a < N) {
      uint32_t ia = rowptr[a], ea = rowptr[a + 1], ib = 0, eb = 0;
      if (b < N) {
        ib = rowptr[b];
        eb = rowptr[b + 1];
      }
      while (ia < ea || ib < eb) {
        const uint32_t ca = ia < ea ? col[ia] : 0xffffffffu, cb = ib < eb ? col[ib] : 0xffffffffu;
        if (ca <= cb) ia++;
        if (cb <= ca) ib++;
        n++;
      }
    }
    if (n) {
      atomicMax(tw + t, n);
      atomicMax(maxes + 3, n);
    }
  }
}

template <int R, bool CPLX, bool PAIRS = false>
__global__ void __launch_bounds__(kPlanBlock)
k_plan_fill(uint32_t N, uint32_t ntiles, const uint32_t *__restrict__ rowptr,
            const uint32_t *__restrict__ col, const double2 *__restrict__ val,
            const uint32_t *__restrict__ ent_begin, const uint32_t *__restrict__ run_begin,
            const uint32_t *__restrict__ tw, const uint32_t *__restrict__ truns,
            const uint32_t *__restrict__ tuniq, uint4 *hdr, uint2 *runs, uint16_t *eslot,
            void *eval) {
  extern __shared__ uint32_t pkeys[];  // [kPlanCap] keys, [kPlanCap] distinct, [kPlanCap] run starts
  uint32_t *uniq = pkeys + kPlanCap;
  uint32_t *rstart = uniq + kPlanCap;
  using Val = typename TiledTypes<CPLX>::Val;
  Val *ev = static_cast<Val *>(eval);
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t r0 = t * R, r1 = min(r0 + R, N);
    const uint32_t e0 = rowptr[r0], T = rowptr[r1] - e0;
    if (T > kPlanCap) continue;  // the count kernel flagged it; the plan is not used
    const uint32_t w = tw[t], nruns = truns[t], nuniq = tuniq[t];
    if (threadIdx.x == 0) hdr[t] = make_uint4(ent_begin[t], run_begin[t], nuniq, w | (nruns << 16));
    const uint32_t n2 = plan_sort_tile(pkeys, col, e0, T, r0, r1);
    // distinct columns and run starts in sorted order
    uint32_t ubase = 0, rbase = 0;
    for (uint32_t b = 0; b < n2; b += blockDim.x) {
      const uint32_t i = b + threadIdx.x;
      const uint32_t f = i < n2 ? plan_flags(pkeys, i) : 0u;
      uint32_t ut, rt;
      const uint32_t up = plan_block_scan(f & 1u, &ut);
      const uint32_t rp = plan_block_scan(f >> 1, &rt);
      if (f & 1u) uniq[ubase + up] = pkeys[i];
      if (f & 2u) rstart[rbase + rp] = ubase + up;
      ubase += ut;
      rbase += rt;
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < nruns; q += blockDim.x) {
      const uint32_t u = rstart[q];
      const uint32_t len = (q + 1 < nruns ? rstart[q + 1] : nuniq) - u;
      runs[run_begin[t] + q] = make_uint2(uniq[u], (u << 16) | len);
    }
    // the shared-memory slot of column c (own rows first, then the runs)
    auto slot_of = [&](uint32_t c) -> uint32_t {
      if (c >= r0 && c < r1) return c - r0;
      uint32_t lo = 0, hi = nuniq;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (uniq[mid] < c) lo = mid + 1; else hi = mid;
      }
      return R + lo;
    };
    if constexpr (PAIRS) {
      // entries: [w][R/2] of {slot | rows << 14} and two values (zero for
      // a row without the column), padding past each pair's merge
      const uint64_t base = (uint64_t)ent_begin[t] * (R / 2);
      for (uint32_t u = threadIdx.x; u < R / 2; u += blockDim.x) {
        const uint32_t a = r0 + 2 * u, b = a + 1;
        uint32_t ia = 0, ea = 0, ib = 0, eb = 0;
        if (a < r1) {
          ia = rowptr[a];
          ea = rowptr[a + 1];
        }
        if (b < r1) {
          ib = rowptr[b];
          eb = rowptr[b + 1];
        }
        for (uint32_t k = 0; k < w; k++) {
          uint16_t slot = kSlotPad;
          Val va{}, vb{};
          if (ia < ea || ib < eb) {
            const uint32_t ca = ia < ea ? col[ia] : 0xffffffffu, cb = ib < eb ? col[ib] : 0xffffffffu;
            const uint32_t c = ca < cb ? ca : cb;
            uint32_t mask = 0;
            if (ca == c) {
              va = val[ia++];
              mask |= 1u;
            }
            if (cb == c) {
              vb = val[ib++];
              mask |= 2u;
            }
            slot = (uint16_t)(slot_of(c) | (mask << 14));
          }
          eslot[base + (uint64_t)k * (R / 2) + u] = slot;
          ev[2 * (base + (uint64_t)k * (R / 2) + u)] = va;
          ev[2 * (base + (uint64_t)k * (R / 2) + u) + 1] = vb;
        }
      }
      __syncthreads();
      continue;
    }
    // entries: [w][R] slots and values, padding past each row's length
    const uint64_t base = (uint64_t)ent_begin[t] * R;
    for (uint32_t it = threadIdx.x; it < w * R; it += blockDim.x) {
      const uint32_t k = it / R, lr = it % R;
      uint16_t slot = kSlotPad;
      Val v{};
      const uint32_t r = r0 + lr;
      if (r < r1) {
        const uint32_t rb = rowptr[r], re = rowptr[r + 1];
        if (rb + k < re) {
          slot = (uint16_t)slot_of(col[rb + k]);
          const double2 a = val[rb + k];
          if constexpr (CPLX) v = a;
          else v = a.x;
        }
      }
      eslot[base + (uint64_t)k * R + lr] = slot;
      ev[base + (uint64_t)k * R + lr] = v;
    }
    __syncthreads();
  }
}

}  // namespace tbtkkpm
