// Launch wrappers and the dispatch table of the recursion-step kernels.
// Each table entry is one compiled configuration (vector type, threads per
// row TPR, values per thread VPT, register cap MINB); the driver or the
// autotuner picks an entry per batch shape.
#pragma once

#include "kpm_async.cuh"
#include "kpm_bulk.cuh"
#include "kpm_real.cuh"
#include "kpm_tiled.cuh"
#include "kpm_host.h"
#include "kpm_kernels.cuh"

#include <algorithm>

namespace tbtkkpm {

// Vector classes of the step kernels (Real: real float vectors of a real
// matrix at mixed precision, see kpm_real.cuh).
enum StepClass : int {
  kClassFP64 = 0,
  kClassMixed = 1,
  kClassMixedDots = 2,
  kClassMixedReal = 3,
  kClassMixedRealDots = 4
};

struct StepArgs {
  Sell A;
  uint32_t Bp;
  const void *x;
  void *y;
  Targets tg;
  uint32_t n_out;
  double2 *dots;
  int *err;  // device flag set by a bounded wait that ran out (bulk kernels)
  const TilePlan *plan = nullptr;  // tile-staged steps: the matrix's plan for their R
  uint32_t wait_limit = kWaitLimit;  // polls per staged-row wait (tile-staged steps)
};

// Launches one step with a grid of min(tiles, resident blocks, max_grid)
// blocks and returns the grid used (the caller sizes per-block buffers).
using StepFn = void (*)(cudaStream_t, int device, unsigned max_grid, const StepArgs &,
                        unsigned *grid);

// variant: the register cap (min blocks per SM, 2-4) of a register-staged
// kernel, or 100 + 10*stages + warps per block of a bulk-copy kernel.
struct StepEntry {
  int cls, tpr, vpt, minb;
  StepFn first, rest;
};

template <typename V, typename AR, int VPT, bool FIRST, bool DOTS, int S, int WPB>
void launch_bulk(cudaStream_t st, int device, unsigned max_grid, const StepArgs &a,
                 unsigned *grid) {
  auto kern = kpm_step_bulk<V, AR, VPT, FIRST, DOTS, S, WPB>;
  constexpr uint32_t smem = bulk_smem_bytes<V, VPT, S, WPB>();
  static int per_sm[64] = {0};
  const int d = device & 63;
  if (per_sm[d] == 0) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * WPB, smem) != cudaSuccess ||
        nb < 1) {
      cudaGetLastError();
      nb = 1;
    }
    per_sm[d] = nb;
  }
  const uint64_t rows = (uint64_t)a.A.nslices * 32;
  uint64_t g = std::min<uint64_t>((rows + WPB - 1) / WPB, (uint64_t)per_sm[d] * sm_count(device));
  if (max_grid) g = std::min<uint64_t>(g, max_grid);
  g = std::max<uint64_t>(g, 1);
  *grid = (unsigned)g;
  kern<<<(unsigned)g, 32 * WPB, smem, st>>>(a.A, a.Bp, static_cast<const V *>(a.x),
                                             static_cast<V *>(a.y), a.tg, a.n_out, a.dots, a.err);
}

#define TBTKKPM_BULK_ENTRY(CLS, V, AR, P, D, S, WPB)                                 \
  {CLS, 32, P, 100 + 10 * S + WPB, &launch_bulk<V, AR, P, true, D, S, WPB>,          \
   &launch_bulk<V, AR, P, false, D, S, WPB>}

template <typename V, typename AR, int TPR, int VPT, bool FIRST, bool DOTS, int MINB>
void launch_step(cudaStream_t st, int device, unsigned max_grid, const StepArgs &a,
                 unsigned *grid) {
  auto kern = kpm_step<V, AR, TPR, VPT, FIRST, DOTS, MINB>;
  static int per_sm[64] = {0};
  const int d = device & 63;
  if (per_sm[d] == 0) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kBlock, 0) != cudaSuccess ||
        nb < 1) {
      cudaGetLastError();
      nb = 1;
    }
    per_sm[d] = nb;
  }
  constexpr int RPB = kBlock / TPR;
  const uint64_t tiles = ((uint64_t)a.A.nslices * 32 + RPB - 1) / RPB;
  uint64_t g = std::min<uint64_t>(tiles, (uint64_t)per_sm[d] * sm_count(device));
  if (max_grid) g = std::min<uint64_t>(g, max_grid);
  g = std::max<uint64_t>(g, 1);
  *grid = (unsigned)g;
  kern<<<(unsigned)g, kBlock, 0, st>>>(a.A, a.Bp, static_cast<const V *>(a.x),
                                       static_cast<V *>(a.y), a.tg, a.n_out, a.dots);
}

#define TBTKKPM_STEP_ENTRY(CLS, V, AR, T, P, D, MB)                                 \
  {CLS, T, P, MB, &launch_step<V, AR, T, P, true, D, MB>,                           \
   &launch_step<V, AR, T, P, false, D, MB>}

template <int TPR, int VPT, bool FIRST, bool DOTS, int MINB, int G, int OPT = 0>
void launch_real(cudaStream_t st, int device, unsigned max_grid, const StepArgs &a,
                 unsigned *grid) {
  auto kern = kpm_step_real<TPR, VPT, FIRST, DOTS, MINB, G, OPT>;
  // dot-product sums in shared memory (OPT bit 3)
  constexpr uint32_t smem = (DOTS && (OPT & 8)) ? 2u * VPT * kBlock * 8u : 0u;
  static int per_sm[64] = {0};
  const int d = device & 63;
  if (per_sm[d] == 0) {
    if (smem) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kBlock, smem) != cudaSuccess ||
        nb < 1) {
      cudaGetLastError();
      nb = 1;
    }
    per_sm[d] = nb;
  }
  constexpr int RPB = kBlock / TPR;
  const uint64_t tiles = ((uint64_t)a.A.nslices * 32 + RPB - 1) / RPB;
  uint64_t g = std::min<uint64_t>(tiles, (uint64_t)per_sm[d] * sm_count(device));
  if (max_grid) g = std::min<uint64_t>(g, max_grid);
  g = std::max<uint64_t>(g, 1);
  *grid = (unsigned)g;
  kern<<<(unsigned)g, kBlock, smem, st>>>(a.A, a.Bp, static_cast<const float *>(a.x),
                                          static_cast<float *>(a.y), a.tg, a.n_out, a.dots);
}

// variant MB + 10*G: register cap MB, G entries gathered per round trip
// (G 0: the default for the shape)
#define TBTKKPM_REAL_ENTRY(CLS, T, P, D, MB, G)                                     \
  {CLS, T, P, MB + 10 * G, &launch_real<T, P, true, D, MB, G>,                      \
   &launch_real<T, P, false, D, MB, G>}
// variant MB + 100*OPT: the OPT bits of kpm_step_real
#define TBTKKPM_REAL_ENTRY_OPT(CLS, T, P, D, MB, OPT)                               \
  {CLS, T, P, MB + 100 * OPT, &launch_real<T, P, true, D, MB, 0, OPT>,              \
   &launch_real<T, P, false, D, MB, 0, OPT>}

template <int VPT, bool FIRST, bool DOTS, int S, int WMAX, int WPB>
void launch_async(cudaStream_t st, int device, unsigned max_grid, const StepArgs &a,
                  unsigned *grid) {
  auto kern = kpm_step_async<VPT, FIRST, DOTS, S, WMAX, WPB>;
  constexpr uint32_t smem = async_smem_bytes<VPT, S, WMAX, WPB>();
  static int per_sm[64] = {0};
  const int d = device & 63;
  if (per_sm[d] == 0) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * WPB, smem) != cudaSuccess ||
        nb < 1) {
      cudaGetLastError();
      nb = 1;
    }
    per_sm[d] = nb;
  }
  const uint64_t tiles = ((uint64_t)a.A.nslices * 32 + WPB - 1) / WPB;
  uint64_t g = std::min<uint64_t>(tiles, (uint64_t)per_sm[d] * sm_count(device));
  if (max_grid) g = std::min<uint64_t>(g, max_grid);
  g = std::max<uint64_t>(g, 1);
  *grid = (unsigned)g;
  kern<<<(unsigned)g, 32 * WPB, smem, st>>>(a.A, a.Bp, static_cast<const float2 *>(a.x),
                                             static_cast<float2 *>(a.y), a.tg, a.n_out, a.dots);
}

// variant 10000 + 1000*S + 10*WMAX + WPB: the cp.async-staged kernel with S
// stages of WMAX gathered rows per warp, WPB warps per block
#define TBTKKPM_ASYNC_ENTRY(CLS, P, D, S, WMAX, WPB)                                \
  {CLS, 32, P, 10000 + 1000 * S + 10 * WMAX + WPB,                                 \
   &launch_async<P, true, D, S, WMAX, WPB>, &launch_async<P, false, D, S, WMAX, WPB>}

// Tile-staged step variants: 100000 + 1000000*CV + 1000*R + 10*CW + BPS
// (CV the widening split of kpm_step_tiled, plus 100 for the row-pair
// form, R rows per tile, CW consumer warps, BPS blocks per SM).
constexpr int kTiledVariant = 100000;
inline bool is_tiled_variant(int v) { return v >= kTiledVariant; }
inline int tiled_rows(int v) { return ((v - kTiledVariant) % 1000000) / 1000; }
inline bool tiled_pairs(int v) { return (v - kTiledVariant) / 1000000 >= 100; }
inline int tiled_bps(int v) { return v % 10; }

template <bool CPLX, int TPR, int VPT, int R, int CW, int BPS, bool FIRST, bool DOTS, int CV,
          bool F64 = false>
void launch_tiled(cudaStream_t st, int device, unsigned max_grid, const StepArgs &a,
                  unsigned *grid) {
  using E = typename TiledTypes<CPLX, F64>::E;
  using Val = typename TiledTypes<CPLX, F64>::Val;
  auto kern = kpm_step_tiled<CPLX, TPR, VPT, R, CW, BPS, FIRST, DOTS, CV, F64>;
  *grid = 0;
  if (!a.plan || a.plan->R != (uint32_t)R || a.plan->pairs != (CV >= 100 ? 1u : 0u)) return;
  const TilePlan &p = *a.plan;
  const TiledLayout ly =
      tiled_layout(p, a.Bp * (uint32_t)sizeof(E), (uint32_t)sizeof(Val), tiled_budget(BPS));
  if (ly.stages == 0) return;
  static bool attr[64] = {false};
  const int d = device & 63;
  if (!attr[d]) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tiled_budget(BPS));
    attr[d] = true;
  }
  uint64_t g = std::min<uint64_t>(p.ntiles, (uint64_t)BPS * sm_count(device));
  if (max_grid) g = std::min<uint64_t>(g, max_grid);
  g = std::max<uint64_t>(g, 1);
  *grid = (unsigned)g;
  // the ring holds the block's dot-product reduction at the end (2 doubles
  // per consumer thread)
  const uint32_t smem = kTiledHeader + std::max(ly.stages * ly.stage_bytes, 32u * CW * 16u);
  kern<<<(unsigned)g, 32 * (CW + 1), smem, st>>>(
      p, ly, a.Bp, static_cast<const E *>(a.x), static_cast<E *>(a.y), a.tg, a.n_out, a.dots,
      a.err, a.wait_limit);
}

#define TBTKKPM_TILED_ENTRY(CLS, CPLX, T, P, D, R, CW, BPS, CV)                     \
  {CLS, T, P, kTiledVariant + 1000000 * CV + 1000 * R + 10 * CW + BPS,               \
   &launch_tiled<CPLX, T, P, R, CW, BPS, true, D, CV>,                               \
   &launch_tiled<CPLX, T, P, R, CW, BPS, false, D, CV>}
// the FP64 recursion on complex128 vectors (kClassFP64)
#define TBTKKPM_TILED_ENTRY_F64(CLS, T, P, R, CW, BPS)                              \
  {CLS, T, P, kTiledVariant + 1000 * R + 10 * CW + BPS,                              \
   &launch_tiled<true, T, P, R, CW, BPS, true, false, 0, true>,                      \
   &launch_tiled<true, T, P, R, CW, BPS, false, false, 0, true>}

extern const StepEntry kStepsFP64[];
extern const int kNumStepsFP64;
extern const StepEntry kStepsMixed[];
extern const int kNumStepsMixed;
extern const StepEntry kStepsMixedDots[];
extern const int kNumStepsMixedDots;
extern const StepEntry kStepsMixedReal[];
extern const int kNumStepsMixedReal;
extern const StepEntry kStepsMixedRealDots[];
extern const int kNumStepsMixedRealDots;

}  // namespace tbtkkpm
