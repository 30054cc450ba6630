// Multi-model recursion: one launch advances every active model of a server
// (or an uneven batch of models) by one Chebyshev step.
//
// Each model keeps its own SELL matrix and its own pair of complex64 vector
// buffers [rows][W] (W = the model's lane width).  A lane is one LDOS
// request site: it joins at a step boundary with j_0 = e_site in its column
// and runs its own local step count, so requests enter and leave while the
// others keep going (continuous batching).  A lane whose local step is 1
// takes j_1 = H~ j_0 (the reference's first step,
// Lib/src/Solver/ChebyshevExpander.cpp:159-169); every later step takes
// j_{n+1} = 2H~ j_n - j_{n-1} (:171-186).  The per-element arithmetic is
// the single-model kernel's (entry order, FMA, one rounding to complex64),
// so a lane's direct moments do not depend on the other lanes or models.
//
// The doubling dot products <j_n|j_n> and Re<j_n|j_{n-1}> are accumulated
// in 64-bit fixed point (2^-61 units): every term is one complex64 product
// rounded once to FP32 and then to the fixed-point grid, and integer sums
// are associative, so the moments of a lane are bit-identical whatever the
// grid, the launch configuration, the tile schedule or the other models in
// the launch.  |terms| and all partial sums stay below 1 (||j_n|| <= 1 for
// a spectrum inside [-1, 1]), so 2^61 leaves headroom of 4.
#pragma once

#include "kpm_kernels.cuh"
#include <algorithm>
#include <utility>
#include <vector>

namespace tbtkkpm {

constexpr int32_t kLaneIdle = INT32_MIN / 2;  // base step of a lane without a request
constexpr float kFixScale = 2305843009213693952.0f;  // 2^61
constexpr double kFixUnit = 1.0 / 2305843009213693952.0;  // 2^-61

// One model of a launch (device resident, rebuilt by the host per tick).
struct MultiModel {
  Sell A;                    // model-local SELL, 2H/s
  float2 *vec[2];            // [nslices*32][W]; step n reads vec[(n+1)&1], writes vec[n&1]
  const uint32_t *bitmap;    // rows that are some lane's site
  const uint32_t *trow;      // sorted target rows
  const uint32_t *tcol;      // lane of each target
  uint32_t tcount;
  const int32_t *base;       // [W] global step of the lane's local step 0, or kLaneIdle
  const uint32_t *lane_M;    // [W] moments the lane's request asks for
  long long *dots;           // [2][W] fixed-point sums of the current step
  double2 *mu;               // [W][Mmax] doubled moments (0 and 1 seeded)
  double2 *mu_direct;        // [W][ld] directly gathered moments
  uint32_t tile0;            // first tile of this model in the launch
  uint32_t ntiles;
  double2 *pmu;              // [W][mmax] moments of Green's-function pairs (pair entries)
  uint32_t mmax;
  // tile-staged steps (kpm_multi_tiled.cuh): the model's gather plan for the
  // launch's rows per tile, and the offset of its runs in the launch's run list
  const uint4 *p_hdr;
  const uint2 *p_runs;
  const uint16_t *p_slot;
  const void *p_val;
  uint32_t p_nruns, run0;
};

// A model's target list pairs a row with an entry word: bits 0-7 the lane
// (the column of the vectors), and with kPairEntry set the moment of the
// lane's local step n goes to row n of pair slot (bits 8-15) of pmu, for
// n < the lane's M, instead of row n < ld of the lane's direct-moment row.
constexpr uint32_t kLaneBits = 0xffu;
constexpr uint32_t kPairEntry = 1u << 31;
// lane_M flag of a lane whose request gathers every moment directly
// (Green's-function pairs with to != from): it runs M - 1 steps; the
// doubling sums of its own source still give its error estimate.
constexpr uint32_t kDirectLane = 1u << 31;
constexpr uint32_t kLaneMBits = ~kDirectLane;

// Destination of the moment of local step nl for target entry tc of model
// md, or nullptr when the entry takes no moment at this step.
__device__ __forceinline__ double2 *multi_target_dst(const MultiModel *__restrict__ md, uint32_t tc,
                                                     int32_t nl, uint32_t ld) {
  if (nl < 1) return nullptr;
  const uint32_t c = tc & kLaneBits;
  if (tc & kPairEntry) {
    if ((uint32_t)nl >= (__ldg(md->lane_M + c) & kLaneMBits)) return nullptr;
    return md->pmu + (uint64_t)((tc >> 8) & kLaneBits) * md->mmax + nl;
  }
  if ((uint32_t)nl >= ld) return nullptr;
  return md->mu_direct + (uint64_t)c * ld + nl;
}

// Per-tick launch header (device resident): the models, their tile total,
// the global step of step offset 0 and the model of every tile.
struct MultiHeader {
  uint32_t nmodels;
  uint32_t total_tiles;
  int32_t n_base;
  const uint32_t *tile_model;  // [total_tiles]
  // tile-staged steps (kpm_multi_tiled.cuh): every tile's 96-byte
  // descriptor, the launch's run list, and the tiles a block takes in a row
  const uint4 *tile_desc;
  const uint2 *tile_runs;
  uint32_t run;
  // steps of the tick done so far, when the tick replays a captured graph
  // of one step (kpm_multi_advance ends each replay); null otherwise
  const int32_t *step;
};

// Global step of a launch: the tick's base, the launch's step offset and,
// in a graph replay, the device counter of steps done.
__device__ __forceinline__ int32_t multi_step_index(const MultiHeader *__restrict__ hdr,
                                                    uint32_t step_offset) {
  return hdr->n_base + (int32_t)step_offset + (hdr->step ? *hdr->step : 0);
}

// Ends one replay of a tick's step graph: the next replay is the next step.
static __global__ void kpm_multi_advance(int32_t *step) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *step += 1;
}

// Changes the row stride of a lane buffer [N][W] -> [N][W2] in place for
// rows [r0, r1): lane c < min(W, W2) of row r moves from r W + c to
// r W2 + c, lanes [W, W2) of a widened row are zero.  A launch may only
// cover rows whose source and destination ranges do not overlap those of
// rows still to move (lane_relayout_ranges), so its threads need no order.
template <typename T>
static __global__ void kpm_lane_relayout(T *__restrict__ v, uint32_t r0, uint32_t r1, uint32_t W,
                                         uint32_t W2) {
  const uint64_t n = (uint64_t)(r1 - r0) * W2;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t r = r0 + i / W2;
    const uint32_t c = (uint32_t)(i % W2);
    T x{};
    if (c < W) x = v[r * W + c];
    v[r * W2 + c] = x;
  }
}

// The launches of an in-place restride [N][W] -> [N][W2] (powers of two),
// as row ranges in launch order.  Widening (W2 = W 2^k) moves rows from the
// end: rows [a, b) with a 2^k >= b read [a W, b W) and write [a W2, b W2),
// which lie above every row not yet moved; row 0 goes last (its lanes
// c < W stay in place).  Narrowing (W = W2 2^k) moves rows from the start:
// rows [a, b) with b <= a 2^k write below their own sources and above the
// rows already moved; row 0 stays.
inline void lane_relayout_ranges(uint32_t N, uint32_t W, uint32_t W2,
                                 std::vector<std::pair<uint32_t, uint32_t>> &out) {
  out.clear();
  if (W == W2 || N == 0) return;
  if (W2 > W) {
    const uint32_t f = W2 / W;
    for (uint32_t b = N; b > 0;) {
      const uint32_t a = b == 1 ? 0 : (uint32_t)(((uint64_t)b + f - 1) / f);
      out.push_back({a, b});
      b = a;
    }
  } else {
    const uint64_t f = W / W2;
    for (uint32_t a = 1; a < N;) {
      const uint32_t b = (uint32_t)std::min<uint64_t>(N, (uint64_t)a * f);
      out.push_back({a, b});
      a = b;
    }
  }
}

// A block takes runs of kRun consecutive tiles (run r, r + gridDim.x, ...),
// so it changes model (and flushes its sums) at most once per run.
constexpr uint32_t kRun = 8;

// Fills the tile -> model map of a launch: one block per model.
static __global__ void kpm_multi_tilemap(const MultiModel *__restrict__ models,
                                         const MultiHeader *__restrict__ hdr, uint32_t *tile_model) {
  if (blockIdx.x >= hdr->nmodels) return;
  const uint32_t t0 = models[blockIdx.x].tile0, nt = models[blockIdx.x].ntiles;
  for (uint32_t t = threadIdx.x; t < nt; t += blockDim.x) tile_model[t0 + t] = blockIdx.x;
}

// Adds a thread's fixed-point sums (msum[j][tid] for <j|j>, msum[VPT + j]
// for <j|j_prev>) into the model's dots: a sum over the warp's threads of
// the same columns, then one atomic per column and warp; clears the sums.
template <typename P, int VPT, int TPR>
__device__ __forceinline__ void multi_flush(long long (*msum)[kBlock], long long *dots,
                                            uint32_t W, int sub) {
#pragma unroll
  for (int j = 0; j < VPT; j++) {
    long long a = msum[j][threadIdx.x], b = msum[VPT + j][threadIdx.x];
#pragma unroll
    for (int off = TPR; off < 32; off <<= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, off);
      b += __shfl_xor_sync(0xffffffffu, b, off);
    }
    if ((threadIdx.x & 31) < TPR) {
      const uint32_t c = P::col_of(sub, j);
      if (a) atomicAdd(reinterpret_cast<unsigned long long *>(dots + c), (unsigned long long)a);
      if (b) atomicAdd(reinterpret_cast<unsigned long long *>(dots + W + c), (unsigned long long)b);
    }
    msum[j][threadIdx.x] = msum[VPT + j][threadIdx.x] = 0;
  }
}

// One recursion step for every model of the launch.  Blocks take runs of
// the concatenated tiles (kBlock/TPR rows each) of all models; a tile's row
// fetch is issued one tile ahead as in kpm_step.
template <int TPR, int VPT, int MINB>
__global__ void __launch_bounds__(kBlock, MINB)
kpm_multi_step(const MultiModel *__restrict__ models, const MultiHeader *__restrict__ hdr,
               uint32_t step_offset, uint32_t W, uint32_t ld) {
  using V = float2;
  using AR = Wide64;
  using P = Pack<V, TPR, VPT>;
  using L = typename P::L;
  using Acc = double2;
  using Val = double2;
  constexpr int NL = P::NL;
  constexpr int G = entries_in_flight<V, VPT, MINB>();
  constexpr int PF = TPR == 1 ? G : 1;
  const int sub = threadIdx.x % TPR;
  const int grp = threadIdx.x / TPR;
  const unsigned mask = 0xffffffffu;
  const uint32_t nmodels = hdr->nmodels, total = hdr->total_tiles;
  const uint32_t *__restrict__ tile_model = hdr->tile_model;
  const int32_t n = multi_step_index(hdr, step_offset);
  if (nmodels == 0) return;

  // per-thread fixed-point sums in shared memory (see multi_flush)
  __shared__ long long msum[2 * VPT][kBlock];
#pragma unroll
  for (int j = 0; j < 2 * VPT; j++) msum[j][threadIdx.x] = 0;

  // the model of the tile being computed and of the one being fetched
  uint32_t mi = kPad, fi = kPad;
  Sell A{}, FA{};
  const float2 *x = nullptr;
  float2 *y = nullptr;
  const float2 *fy = nullptr;
  uint32_t ft0 = 0;    // first tile of the fetched tile's model
  uint32_t first = 0;  // bit j: lane of value j is at its local step 1
  // fields of the current model kept in registers
  const uint32_t *t_bitmap = nullptr, *t_row = nullptr, *t_col = nullptr;
  const int32_t *t_base = nullptr;
  long long *t_dots = nullptr;
  uint32_t t_count = 0;

  // model and slice bounds of the row a thread takes in tile w (issued a tile
  // before the row's entries, which depend on them)
  auto bounds_of = [&](uint32_t w, uint32_t &model) -> RowBounds {
    model = __ldg(tile_model + w);
    const MultiModel *q = models + model;
    Sell s{};
    s.slice_ptr = q->A.slice_ptr;
    s.nslices = q->A.nslices;
    return load_bounds<TPR>(s, w - q->tile0, grp);
  };
  auto fetch = [&](uint32_t w, uint32_t i, RowBounds b, RowFetch<V, AR, TPR, VPT, PF> &f) {
    if (i != fi) {
      fi = i;
      const MultiModel *q = models + i;
      FA.slice_ptr = q->A.slice_ptr;
      FA.col = q->A.col;
      FA.val = q->A.val;
      FA.N = q->A.N;
      FA.nslices = q->A.nslices;
      fy = q->vec[n & 1];
      ft0 = q->tile0;
    }
    fetch_row<V, AR, TPR, VPT, PF, false>(FA, W, fy, w - ft0, grp, sub, b, f);
  };
  // the tile after w in this block's order
  auto next_tile = [&](uint32_t w) -> uint32_t {
    const uint32_t nw = w + 1;
    if (nw % kRun != 0) return nw;
    return (w / kRun + gridDim.x) * kRun;
  };

  RowFetch<V, AR, TPR, VPT, PF> cur, nxt;
  uint32_t cur_model = 0, nxt_model = 0;
  uint32_t w = blockIdx.x * kRun;
  if (w < total) {
    const RowBounds b0 = bounds_of(w, cur_model);
    fetch(w, cur_model, b0, cur);
  }
  uint32_t wn = next_tile(w), bm = 0;  // next tile, its model and bounds
  RowBounds bb{0, 0};
  if (wn < total) bb = bounds_of(wn, bm);
  for (; w < total; w = wn, wn = next_tile(wn)) {
    if (cur_model != mi) {
      // block-uniform: every thread of the block is on the same tile
      if (mi != kPad) multi_flush<P, VPT, TPR>(msum, t_dots, W, sub);
      mi = cur_model;
      const MultiModel *md = models + mi;
      A.slice_ptr = md->A.slice_ptr;
      A.col = md->A.col;
      A.val = md->A.val;
      A.N = md->A.N;
      A.nslices = md->A.nslices;
      x = md->vec[(n + 1) & 1];
      y = md->vec[n & 1];
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
      const uint32_t row = cur.row, l = cur.l, cb = cur.cb, ce = cur.ce, wd = ce - cb;
      Acc acc[VPT];
      L yv[NL];
      row_y(cur, y, W, sub, yv);
#pragma unroll
      for (int j = 0; j < VPT; j++) {
        if ((first >> j) & 1u) {
          acc[j] = Acc{0, 0};
        } else {
          const Acc v = cur.live ? pack_get<P, Acc>(yv, j) : Acc{0, 0};
          acc[j] = Acc{-v.x, -v.y};
        }
      }
      if constexpr (TPR == 1) {
        for (uint32_t kb = 0; kb < wd; kb += G) {
          uint32_t cc[G];
          Val vv[G];
          L raw[G][NL];
#pragma unroll
          for (int g = 0; g < G; g++)
            cc[g] = kb == 0 ? cur.cc[g]
                            : ((kb + g < wd) ? __ldcs(A.col + (uint64_t)(cb + kb + g) * 32 + l) : kPad);
#pragma unroll
          for (int g = 0; g < G; g++)
            if (cc[g] != kPad) {
              vv[g] = AR::value(A, (uint64_t)(cb + kb + g) * 32 + l);
              P::load(x + (uint64_t)cc[g] * W, sub, raw[g]);
            }
#pragma unroll
          for (int g = 0; g < G; g++) {
            if (cc[g] == kPad) continue;
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = AR::mac(acc[j], vv[g], pack_get<P, Acc>(raw[g], j));
          }
        }
      } else {
        for (uint32_t kb = 0; kb < wd; kb += TPR) {
          uint32_t myc;
          Val myv;
          if (kb == 0) {
            myc = cur.cc[0];
            myv = cur.vv[0];
          } else {
            myc = kPad;
            myv = Val{0, 0};
            if (kb + sub < wd) {
              myc = __ldcs(A.col + (uint64_t)(cb + kb + sub) * 32 + l);
              if (myc != kPad) myv = AR::value(A, (uint64_t)(cb + kb + sub) * 32 + l);
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
              const int src = (int)min(j0 + g, nk - 1);
              Val v;
              v.x = __shfl_sync(mask, myv.x, src, TPR);
              v.y = __shfl_sync(mask, myv.y, src, TPR);
              if (cc[g] == kPad) continue;
#pragma unroll
              for (int j = 0; j < VPT; j++) acc[j] = AR::mac(acc[j], v, pack_get<P, Acc>(raw[g], j));
            }
          }
        }
      }
      if (cur.live) {
        // first-step lanes: j_1 = (1/2)(2H~) j_0, an exact halving of the
        // same accumulation
#pragma unroll
        for (int j = 0; j < VPT; j++)
          if ((first >> j) & 1u) acc[j] = AR::half(acc[j]);
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
                if (j == jt) *dst = acc[j];
            }
          }
        }
        float2 af[VPT];
#pragma unroll
        for (int j = 0; j < VPT; j++)
          af[j] = make_float2(__double2float_rn(acc[j].x), __double2float_rn(acc[j].y));
        P::storef(y + (uint64_t)row * W, sub, af);
        L self[NL];
        P::load(x + (uint64_t)row * W, sub, self);
#pragma unroll
        for (int j = 0; j < VPT; j++) {
          const float2 b = P::getf(self, j);
          msum[j][threadIdx.x] += __float2ll_rn(fmaf(af[j].x, af[j].x, af[j].y * af[j].y) * kFixScale);
          msum[VPT + j][threadIdx.x] += __float2ll_rn(fmaf(af[j].x, b.x, af[j].y * b.y) * kFixScale);
        }
      }
    }
    cur = nxt;
    cur_model = nxt_model;
  }
  if (mi != kPad) multi_flush<P, VPT, TPR>(msum, t_dots, W, sub);
}

// After a step: the doubled moments of every active lane,
// mu_{2m} = 2<j_m|j_m> - mu_0 and mu_{2m-1} = 2<j_m|j_{m-1}> - mu_1 for the
// lane's local step m, and the fixed-point sums cleared for the next step.
// One block per model, one thread per lane.
static __global__ void kpm_multi_finalize(const MultiModel *__restrict__ models,
                                   const MultiHeader *__restrict__ hdr, uint32_t step_offset,
                                   uint32_t W, uint32_t Mmax, uint32_t ld) {
  if (blockIdx.x >= hdr->nmodels) return;
  const MultiModel *md = models + blockIdx.x;
  const int32_t n = multi_step_index(hdr, step_offset);
  for (uint32_t c = threadIdx.x; c < W; c += blockDim.x) {
    const long long a = md->dots[c], b = md->dots[W + c];
    md->dots[c] = 0;
    md->dots[W + c] = 0;
    const int32_t base = md->base[c];
    if (base == kLaneIdle) continue;
    const int32_t m = n - base;
    const uint32_t M = md->lane_M[c] & kLaneMBits;
    if (m < 1 || (uint32_t)m > M / 2) continue;
    double2 *row = md->mu + (uint64_t)c * Mmax;
    if (m == 1) row[1] = md->mu_direct[(uint64_t)c * ld + 1];
    const double2 mu0 = row[0], mu1 = row[1];
    const double sa = (double)a * kFixUnit, sb = (double)b * kFixUnit;
    if (2 * (uint32_t)m < M) row[2 * m] = make_double2(2.0 * sa - mu0.x, -mu0.y);
    if (m >= 2 && 2 * (uint32_t)m - 1 < M) row[2 * m - 1] = make_double2(2.0 * sb - mu1.x, -mu1.y);
  }
}

// A lane joining at global step g (its local step 1 is computed at g):
// column c of the buffer step g reads as j_0 becomes e_site, its moment rows
// are cleared and mu_0 = <site|site> = 1 is set.
struct MultiJoin {
  float2 *x;          // the model's vec[(g+1)&1]
  double2 *mu;        // the lane's row of mu [Mmax]
  double2 *mu_direct; // the lane's row of mu_direct [ld]
  uint32_t rows;      // model rows (N)
  uint32_t col, site;
  uint32_t W;         // the model's lane width
  uint32_t real;      // the model's vectors are real floats (x holds float)
  float2 *x_prev;     // the model's vec[g&1] (column cleared when not null)
  uint32_t M;         // moments of the lane's request
};

static __global__ void kpm_multi_join(const MultiJoin *__restrict__ joins, uint32_t Mmax, uint32_t ld) {
  const MultiJoin jn = joins[blockIdx.y];
  const uint32_t W = jn.W;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < jn.rows; r += stride) {
    if (jn.real) {
      reinterpret_cast<float *>(jn.x)[r * W + jn.col] = r == jn.site ? 1.0f : 0.0f;
      if (jn.x_prev) reinterpret_cast<float *>(jn.x_prev)[r * W + jn.col] = 0.0f;
    } else {
      jn.x[r * W + jn.col] = r == jn.site ? make_float2(1.0f, 0.0f) : make_float2(0.0f, 0.0f);
      if (jn.x_prev) jn.x_prev[r * W + jn.col] = make_float2(0.0f, 0.0f);
    }
  }
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < Mmax; k += stride) {
    jn.mu[k] = make_double2(k == 0 ? 1.0 : 0.0, 0.0);
    if (k < ld) jn.mu_direct[k] = make_double2(k == 0 ? 1.0 : 0.0, 0.0);
  }
}

// The moments of a finished request, [K][M] contiguous: the direct moments
// for n <= M/2 and the doubled ones above, damped by a[n]/b as kpm_damp
// (raw copies of both kinds when raw and raw_direct are not null).
struct MultiDone {
  const double2 *mu;        // lane row [Mmax]
  const double2 *mu_direct; // lane row [ld]
};

static __global__ void kpm_multi_prepare(const MultiDone *__restrict__ lanes, uint32_t K, uint32_t M,
                                  const double *__restrict__ a, double b, int damp,
                                  double2 *__restrict__ out, double2 *__restrict__ raw,
                                  double2 *__restrict__ raw_direct) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint64_t)K * M) return;
  const uint32_t k = (uint32_t)(i / M), nn = (uint32_t)(i % M);
  const uint32_t half = M / 2;
  const MultiDone d = lanes[k];
  const double2 dbl = d.mu[nn];
  if (raw) raw[i] = dbl;
  double2 c = dbl;
  if (nn <= half) {
    c = d.mu_direct[nn];
    if (raw_direct) raw_direct[(uint64_t)k * (half + 1) + nn] = c;
  }
  if (damp) {
    const double an = a[nn];
    c = make_double2(__ddiv_rn(__dmul_rn(c.x, an), b), __ddiv_rn(__dmul_rn(c.y, an), b));
  }
  out[i] = c;
}

// Error estimate of each finished lane, the single-model doubling_error on
// the device: 4 sqrt(2) max_{2 <= n <= M/2} |mu_n - mu_direct_n| divided by
// max_{n < M} |mu_n| (mu the doubled row).  One block of kErrorBlock
// threads per lane; maxima do not depend on the reduction order.
constexpr int kErrorBlock = 256;
static __global__ void __launch_bounds__(kErrorBlock)
kpm_multi_error(const MultiDone *__restrict__ lanes, uint32_t M, double *__restrict__ err) {
  __shared__ double rs[kErrorBlock], rd[kErrorBlock];
  const MultiDone d = lanes[blockIdx.x];
  const uint32_t ld = M / 2 + 1;
  double sc = 0.0, dm = 0.0;
  for (uint32_t n = threadIdx.x; n < M; n += kErrorBlock) {
    const double2 a = d.mu[n];
    sc = fmax(sc, hypot(a.x, a.y));
    if (n >= 2 && n < ld) {
      const double2 b = d.mu_direct[n];
      dm = fmax(dm, hypot(a.x - b.x, a.y - b.y));
    }
  }
  rs[threadIdx.x] = sc;
  rd[threadIdx.x] = dm;
  __syncthreads();
  for (int h = kErrorBlock / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      rs[threadIdx.x] = fmax(rs[threadIdx.x], rs[threadIdx.x + h]);
      rd[threadIdx.x] = fmax(rd[threadIdx.x], rd[threadIdx.x + h]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) err[blockIdx.x] = rs[0] > 0 ? 4.0 * sqrt(2.0) * rd[0] / rs[0] : 0.0;
}

// A (to, from) pair of a finished Green's-function request whose lanes
// gathered every moment directly: its moment row in pmu (rows n >= 1
// written by the steps), mu_0 = <to|from>, and the diagonal moment rows of
// its source lane (doubled and direct), which give the error estimate.
struct MultiPair {
  const double2 *row;         // pair slot row [Mmax]
  double mu0;                 // 1 if to == from, else 0
  const double2 *lane_mu;     // the source lane's doubled moments [Mmax]
  const double2 *lane_direct; // its directly gathered moments [ld]
};

// The damped moments of K pairs, [K][M] contiguous (as kpm_multi_prepare).
static __global__ void kpm_multi_prepare_pairs(const MultiPair *__restrict__ pairs, uint32_t K,
                                               uint32_t M, const double *__restrict__ a, double b,
                                               int damp, double2 *__restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint64_t)K * M) return;
  const uint32_t k = (uint32_t)(i / M), nn = (uint32_t)(i % M);
  const MultiPair p = pairs[k];
  double2 c = nn == 0 ? make_double2(p.mu0, 0.0) : p.row[nn];
  if (damp) {
    const double an = a[nn];
    c = make_double2(__ddiv_rn(__dmul_rn(c.x, an), b), __ddiv_rn(__dmul_rn(c.y, an), b));
  }
  out[i] = c;
}

// Error estimate of each pair: the source lane's gap between doubled and
// direct diagonal moments, 4 sqrt(2) max_{2 <= n <= M/2} |mu_n - mu_direct_n|
// (an absolute error scale of moments from these float vectors; the pair's
// own moments are gathered directly, which carry less rounding), relative
// to the pair's max_n |mu_n|.  One block of kErrorBlock threads per pair.
static __global__ void __launch_bounds__(kErrorBlock)
kpm_pair_error(const MultiPair *__restrict__ pairs, uint32_t M, double *__restrict__ err) {
  __shared__ double rs[kErrorBlock], rd[kErrorBlock];
  const MultiPair p = pairs[blockIdx.x];
  const uint32_t ld = M / 2 + 1;
  double sc = threadIdx.x == 0 ? fabs(p.mu0) : 0.0, dm = 0.0;
  for (uint32_t n = threadIdx.x; n < M; n += kErrorBlock) {
    if (n >= 1) {
      const double2 q = p.row[n];
      sc = fmax(sc, hypot(q.x, q.y));
    }
    if (n >= 2 && n < ld) {
      const double2 a = p.lane_mu[n], b = p.lane_direct[n];
      dm = fmax(dm, hypot(a.x - b.x, a.y - b.y));
    }
  }
  rs[threadIdx.x] = sc;
  rd[threadIdx.x] = dm;
  __syncthreads();
  for (int h = kErrorBlock / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      rs[threadIdx.x] = fmax(rs[threadIdx.x], rs[threadIdx.x + h]);
      rd[threadIdx.x] = fmax(rd[threadIdx.x], rd[threadIdx.x + h]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) err[blockIdx.x] = rs[0] > 0 ? 4.0 * sqrt(2.0) * rd[0] / rs[0] : 0.0;
}

}  // namespace tbtkkpm

// ---------------------------------------------------------------- dispatch
#include "kpm_host.h"

namespace tbtkkpm {

// Launch data of the tile-staged steps (ignored by the register-staged
// ones): the shared-memory ring of the launch's class, the device flag a
// staged-row wait that runs out sets, and the polls per wait.
struct MultiLaunch {
  TiledLayout ly;
  int *err;
  uint32_t wait_limit;
};

using MultiFn = void (*)(cudaStream_t, int device, const MultiModel *, const MultiHeader *,
                         uint32_t step_offset, uint32_t W, uint32_t ld, const MultiLaunch &);

// One compiled configuration of a multi-model step for lane width tpr*vpt:
// minb is the register cap of kpm_multi_step(_real), or a tile-staged
// variant code (kTiledVariant + 1000*R + 10*CW + BPS, kpm_multi_tiled.cuh).
struct MultiEntry {
  int tpr, vpt, minb;
  MultiFn launch;
};

// Grid: every resident block of the device (the kernel strides over tiles).
template <int TPR, int VPT, int MINB>
void launch_multi(cudaStream_t st, int device, const MultiModel *models, const MultiHeader *hdr,
                  uint32_t step_offset, uint32_t W, uint32_t ld, const MultiLaunch &) {
  auto kern = kpm_multi_step<TPR, VPT, MINB>;
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
  kern<<<(unsigned)(per_sm[d] * sm_count(device)), kBlock, 0, st>>>(models, hdr, step_offset, W,
                                                                    ld);
}

#define TBTKKPM_MULTI_ENTRY(T, P, MB) {T, P, MB, &launch_multi<T, P, MB>}

extern const MultiEntry kMultiSteps[];
extern const int kNumMultiSteps;

}  // namespace tbtkkpm
