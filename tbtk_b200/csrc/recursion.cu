// The Chebyshev recursion and the energy-grid sums behind the C ABI.
#include "tbtkkpm.h"
#include "kpm_host.h"
#include "kpm_kernels.cuh"
#include "kpm_steps.cuh"
#include "kpm_prefix.cuh"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

namespace tbtkkpm {

namespace {

inline unsigned blocks_for(uint64_t n, unsigned bs = 256) { return (unsigned)((n + bs - 1) / bs); }

// ------------------------------------------------------------ batch shapes
// A batch of B vectors is stored [N][Bp]; a row is owned by TPR threads, each
// holding VPT complex columns (Bp = TPR*VPT >= B).  complex128 batches go up
// to 128 columns (64 B per thread), complex64 batches to 256 (64 B per
// thread).
struct Shape {
  int tpr, vpt;
  int minb = 2;  // variant: register cap + 100 * OPT bits
  uint32_t bp() const { return (uint32_t)(tpr * vpt); }
};

constexpr uint32_t kMaxBatchFP64 = 128;
constexpr uint32_t kMaxBatchMixed = 256;

bool is_mixed(int precision) { return precision != TBTKKPM_FP64; }

// Mixed-precision batches of a real matrix run on real float vectors
// (kpm_real.cuh) unless the caller turned that off.
bool real_mode(const tbtkkpm_matrix *m, int precision) {
  return is_mixed(precision) && m->values_real && m->use_real;
}

// The register-staged shape of a batch (kpm_step / kpm_step_real): the
// fallback of the tile-staged defaults below, and the default of widths the
// tile-staged steps do not serve.
Shape register_shape_for(int precision, uint32_t B, bool real, bool dots) {
  if (real) {
    // a thread per row up to 8 values: it prefetches all of the next row's
    // entries and gathers them in one round (0.51 against 0.71 ms per step
    // for B = 8 on the 2048^2 lattice)
    if (B <= 1) return {1, 1};
    if (B <= 2) return {1, 2};
    if (B <= 4) return {1, 4};
    if (B <= 8) return {1, 8};
    // doubling runs: 16 values per thread with the dot sums in shared
    // memory (variant 802), the fastest register-staged shapes on the
    // 2048^2 lattice at M = 128: 0.84 / 1.83 / 2.91 / 4.93 / 11.9 ms per step
    // for B = 16 / 32 / 64 / 128 / 256
    if (dots) {
      if (B <= 16) return {1, 16, 802};
      if (B <= 32) return {2, 16, 802};
      if (B <= 64) return {4, 16, 802};
      if (B <= 128) return {8, 16, 802};
      return {16, 16, 802};
    }
    // wider batches: the autotuner's choices on the 2048^2 lattice (B = 64:
    // (8, 8) 3.53 ms per step against 5.15 ms for (16, 4))
    if (B <= 16) return {4, 4};
    if (B <= 32) return {4, 8};
    if (B <= 64) return {8, 8};
    if (B <= 128) return {16, 8};
    return {32, 8};
  }
  if (!is_mixed(precision)) {
    if (B <= 1) return {1, 1};
    if (B <= 2) return {2, 1};
    if (B <= 4) return {4, 1};
    if (B <= 8) return {8, 1};
    if (B <= 16) return {16, 1};
    if (B <= 32) return {32, 1};
    if (B <= 64) return {32, 2};
    return {32, 4};
  }
  // complex64 vectors: the fastest compiled shapes on the 2048^2 lattice
  // (B = 4: (1, 4) 0.43 ms per step; B = 64: (8, 8) 5.10 ms against 6.35 ms
  // for (32, 2))
  if (B <= 1) return {1, 1};
  if (B <= 2) return {1, 2};
  if (B <= 4) return {1, 4};
  if (B <= 8) return {4, 2};
  if (B <= 16) return {8, 2};
  if (B <= 32) return {8, 4};
  if (B <= 64) return {8, 8};
  if (B <= 128) return {32, 4};
  return {32, 8};
}

// Tile-staged variant: 100000 + 1000000*CV + 1000*R + 10*CW + BPS.
constexpr int tiled(int cv, int rows, int cw, int bps) {
  return 100000 + 1000000 * cv + 1000 * rows + 10 * cw + bps;
}

// Default shape of a batch.  At mixed precision from 32 sources on (from 16
// for complex vectors) the tile-staged steps are the defaults: ms per step
// measured on the 2048^2 lattice (real float vectors, doubling dots) for
// B = 32 / 64 / 128 / 256: 1.05 / 1.43 / 3.01 / 5.71 against 1.82 / 2.90 /
// 4.79 / 11.8 for the register-staged defaults, and on the 1024^2 Rashba
// lattice (complex64) for B = 16 / 32 / 64 / 128 / 256: 0.38 / 0.55 / 1.09 /
// 2.14 / 4.27 against 1.06 / 1.25 / 1.94 / 3.33 / 8.28.  Without the dots
// (directly gathered moments) the real B = 64 step takes 1.29 ms (0.84 of
// the measured copy bandwidth).  A matrix whose tiles do not fit the ring
// falls back to register_shape_for.
// N: the matrix's rows (0: large).
Shape shape_for(int precision, uint32_t B, bool real = false, bool dots = false, uint32_t N = 0) {
  if (!is_mixed(precision)) {
    // FP64 (complex128 vectors) on the 2048^2 lattice, ms per step for
    // B = 1 / 2 / 4 / 8 / 16: 0.171 / 0.224 / 0.346 / 0.669 / 1.38
    // tile-staged against 0.278 / 0.504 / 0.924 / 2.49 / 4.50
    // register-staged, and for B = 32 / 64 / 128: 2.12 / 4.12 / 8.32
    // (0.96-0.99 of the measured copy bandwidth) against 5.28 / 6.79 / 18.9.
    // Below 2^17 rows a single source is faster register-staged (4.4 against
    // 5.2 us per step at 32k rows); at 32 sources tile staging is as fast or
    // faster from 2k rows on.
    const bool big = N == 0 || N > (1u << 17);
    if (B <= 1 && big) return {1, 1, tiled(0, 64, 2, 8)};
    if (B == 2 && big) return {2, 1, tiled(0, 64, 4, 6)};
    if (B > 2 && B <= 4 && big) return {4, 1, tiled(0, 64, 8, 4)};
    if (B > 4 && B <= 8 && big) return {8, 1, tiled(0, 64, 16, 2)};
    if (B > 8 && B <= 16 && big) return {16, 1, tiled(0, 32, 8, 2)};
    if (B > 16 && B <= 32) return {16, 2, tiled(0, 16, 8, 2)};
    if (B > 32 && B <= 64) return {16, 4, tiled(0, 8, 8, 2)};
    if (B > 64) return {32, 4, tiled(0, 8, 16, 1)};
  }
  if (is_mixed(precision)) {
    // 2-8 sources (rows of 16-64 bytes): small tile-staged blocks, several
    // per SM; doubling LDOS, ms per step for real B = 4 / 8 on the 2048^2
    // lattice 0.167 / 0.237 against 0.347 / 0.505 register-staged (0.0146 /
    // 0.0165 against 0.0186 / 0.0234 at 131k rows), complex B = 2 / 4 / 8 on
    // the 1024^2 Rashba lattice 0.079 / 0.099 / 0.156 against 0.138 / 0.170
    // / 0.383; real B = 16: 0.408 against 0.836 (0.0207 against 0.0267 at
    // 131k rows).  At 2k rows real B = 8 / 16 steps are faster with a
    // register-staged thread per row (10.3 against 12.4 / 13.4 us; about
    // even at 32k rows).
    const bool tiny = N != 0 && N <= (1u << 14);
    if (real) {
      if (B > 2 && B <= 4) return {1, 4, tiled(0, 64, 2, 8)};
      if (B > 4 && B <= 8 && !tiny) return {1, 8, tiled(0, 64, 2, 8)};
      if (B > 8 && B <= 16 && !tiny) return {2, 8, tiled(51, 64, 4, 4)};
    } else {
      if (B == 2) return {1, 2, tiled(0, 64, 2, 6)};
      if (B > 2 && B <= 4) return {2, 2, tiled(0, 64, 4, 6)};
      if (B > 4 && B <= 8) return {2, 4, tiled(0, 64, 4, 4)};
    }
    if (real) {
      if (B > 16 && B <= 32) return {8, 4, tiled(0, 64, 16, 1)};
      if (B > 32 && B <= 64) return {8, 8, tiled(51, 64, 16, 1)};
      if (B > 64 && B <= 128) return {16, 8, tiled(51, 16, 8, 2)};
      if (B > 128) return {32, 8, tiled(51, 16, 16, 1)};
    } else {
      if (B > 8 && B <= 16) return {8, 2, tiled(0, 32, 8, 2)};
      if (B > 16 && B <= 32) return {8, 4, tiled(0, 32, 8, 2)};
      if (B > 32 && B <= 64) return {16, 4, tiled(0, 16, 8, 2)};
      if (B > 64 && B <= 128) return {32, 4, tiled(0, 16, 16, 1)};
      if (B > 128) return {64, 4, tiled(0, 8, 16, 1)};
    }
  }
  return register_shape_for(precision, B, real, dots);
}

int step_class(int precision, bool dots, bool real = false) {
  if (!is_mixed(precision)) return kClassFP64;
  if (real) return dots ? kClassMixedRealDots : kClassMixedReal;
  return dots ? kClassMixedDots : kClassMixed;
}

void step_table(int cls, const StepEntry **t, int *n) {
  if (cls == kClassFP64) {
    *t = kStepsFP64;
    *n = kNumStepsFP64;
  } else if (cls == kClassMixed) {
    *t = kStepsMixed;
    *n = kNumStepsMixed;
  } else if (cls == kClassMixedDots) {
    *t = kStepsMixedDots;
    *n = kNumStepsMixedDots;
  } else if (cls == kClassMixedReal) {
    *t = kStepsMixedReal;
    *n = kNumStepsMixedReal;
  } else {
    *t = kStepsMixedRealDots;
    *n = kNumStepsMixedRealDots;
  }
}

const StepEntry *find_step(int cls, int tpr, int vpt, int minb) {
  const StepEntry *t;
  int n;
  step_table(cls, &t, &n);
  for (int i = 0; i < n; i++)
    if (t[i].tpr == tpr && t[i].vpt == vpt && t[i].minb == minb) return &t[i];
  return nullptr;
}

uint64_t tune_key(int cls, uint32_t Bp) { return ((uint64_t)cls << 32) | Bp; }

// Autotuning results of this process by (device, class, padded width, N,
// nnz): a new handle for a matrix of a tuned shape starts with the tuned
// configuration.
using ShapeKey = std::array<uint64_t, 5>;
std::mutex g_tuned_mu;
std::map<ShapeKey, std::array<int, 3>> g_tuned;

ShapeKey shape_key(const tbtkkpm_matrix *m, int cls, uint32_t Bp) {
  return {(uint64_t)m->device, (uint64_t)cls, Bp, m->N, m->nnz};
}

// The configuration of a batch: a forced entry, the handle's tuned choice
// for this (class, padded width), this process's choice for a matrix of the
// same shape, or the default shape with MINB 2.
const StepEntry *pick_step(const tbtkkpm_matrix *m, int precision, bool dots, uint32_t B,
                           const StepEntry *force) {
  if (force) return force;
  const bool real = real_mode(m, precision);
  const int cls = step_class(precision, dots, real);
  const Shape s = shape_for(precision, B, real, dots, m->N);
  auto it = m->tuned.find(tune_key(cls, s.bp()));
  if (it != m->tuned.end()) {
    const StepEntry *e = find_step(cls, it->second[0], it->second[1], it->second[2]);
    if (e) return e;
  }
  {
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    auto git = g_tuned.find(shape_key(m, cls, s.bp()));
    if (git != g_tuned.end()) {
      const StepEntry *e = find_step(cls, git->second[0], git->second[1], git->second[2]);
      if (e) return e;
    }
  }
  return find_step(cls, s.tpr, s.vpt, s.minb);
}

// A tile-staged entry runs with the matrix's plan for its tile height when
// a ring of at least two stages fits its shared memory.  Otherwise a forced
// entry is refused (TBTKKPM_ERR_UNSUPPORTED, which the autotuner skips) and
// a chosen one gives way to the register-staged default of the batch.
int resolve_tiled(tbtkkpm_matrix *m, int precision, bool dots, uint32_t B, bool forced,
                  const StepEntry *&fn, const TilePlan *&plan) {
  plan = nullptr;
  if (!fn || !is_tiled_variant(fn->minb)) return TBTKKPM_OK;
  const bool cplx = !(fn->cls == kClassMixedReal || fn->cls == kClassMixedRealDots);
  const TilePlan *p = nullptr;
  int rc = tile_plan(m, tiled_rows(fn->minb), cplx, &p, tiled_pairs(fn->minb));
  if (rc) return rc;
  const uint32_t esz = fn->cls == kClassFP64 ? sizeof(double2) : cplx ? sizeof(float2) : sizeof(float);
  const uint32_t vsz = cplx ? sizeof(double2) : sizeof(double);
  if (p && tiled_layout(*p, (uint32_t)(fn->tpr * fn->vpt) * esz, vsz,
                        tiled_budget(tiled_bps(fn->minb))).stages) {
    plan = p;
    return TBTKKPM_OK;
  }
  if (forced)
    return fail(TBTKKPM_ERR_UNSUPPORTED,
                "recursion: the tile-staged step %d x %d / %d does not fit this matrix", fn->tpr,
                fn->vpt, fn->minb);
  const Shape s = register_shape_for(precision, B, !cplx, dots);
  fn = find_step(fn->cls, s.tpr, s.vpt, s.minb);
  return TBTKKPM_OK;
}

// ------------------------------------------------------------ one batch
// The to-indices of a batch (row, batch column, output slot), sorted by row.
struct TargetList {
  std::vector<uint32_t> row, col, out;
};

// Runs the recursion of one batch and leaves the undamped moments in ws.mu
// ([K][M]).  doubling: every source's only target is itself (an LDOS batch);
// the recursion stops at j_{M/2} and the moments come from the doubling
// identities, while the directly gathered moments of steps 0..M/2 land in
// ws.mu_direct ([K][M/2+1]) for the error estimate.  A mixed doubling run
// on a structurally symmetric matrix takes its first steps in FP64 on the
// rows they reach (kpm_prefix) unless `head` is false.
int run_batch(tbtkkpm_matrix *m, int precision, const std::vector<uint32_t> &from,
              const TargetList &tl, uint32_t K, uint32_t M, bool doubling,
              const StepEntry *force = nullptr, bool head = true) {
  Workspace &ws = m->ws;
  cudaStream_t st = m->stream;
  const uint32_t B = (uint32_t)from.size();
  const StepEntry *fn = pick_step(m, precision, doubling, B, force);
  const TilePlan *plan = nullptr;
  int rc0 = resolve_tiled(m, precision, doubling, B, force != nullptr, fn, plan);
  if (rc0) return rc0;
  if (!fn) return fail(TBTKKPM_ERR_UNSUPPORTED, "no recursion kernel for batch %u", B);
  const uint32_t Bp = (uint32_t)(fn->tpr * fn->vpt);
  if (Bp < B) return fail(TBTKKPM_ERR_ARGUMENT, "configuration of %u columns for %u sources", Bp, B);
  const bool real = fn->cls == kClassMixedReal || fn->cls == kClassMixedRealDots;
  const size_t esize = real ? sizeof(float) : (is_mixed(precision) ? sizeof(float2) : sizeof(double2));
  const size_t vbytes = (size_t)m->N * Bp * esize;
  const size_t words = ((size_t)m->N + 31) / 32;
  const uint32_t T = (uint32_t)tl.row.size();
  const uint32_t steps = doubling ? M / 2 : (M >= 2 ? M - 1 : 0);  // last j index computed
  const uint32_t ld_direct = doubling ? steps + 1 : M;
  const unsigned max_grid = (unsigned)sm_count(m->device) * 8;
  int rc;
  if ((rc = ws.vec[0].reserve(vbytes)) || (rc = ws.vec[1].reserve(vbytes)) ||
      (rc = ws.bitmap.reserve(4 * words)) || (rc = ws.tgt.reserve(12 * std::max(T, 1u))) ||
      (rc = ws.from.reserve(4 * std::max(B, 1u))) || (rc = ws.err.reserve(16)) ||
      (rc = ws.mu.reserve(sizeof(double2) * (size_t)std::max(K, 1u) * M)))
    return rc;
  if (doubling &&
      ((rc = ws.mu_direct.reserve(sizeof(double2) * (size_t)std::max(K, 1u) * ld_direct)) ||
       (rc = ws.dots.reserve(sizeof(double2) * 2 * (size_t)Bp * max_grid)) ||
       (rc = ws.col_out.reserve(4 * (size_t)Bp))))
    return rc;
  std::vector<uint32_t> bitmap(words, 0u);
  for (uint32_t r : tl.row) bitmap[r >> 5] |= 1u << (r & 31);
  std::vector<uint32_t> tg_host(3 * (size_t)T);
  std::copy(tl.row.begin(), tl.row.end(), tg_host.begin());
  std::copy(tl.col.begin(), tl.col.end(), tg_host.begin() + T);
  std::copy(tl.out.begin(), tl.out.end(), tg_host.begin() + 2 * (size_t)T);
  cudaError_t e;
  if ((e = cudaMemcpyAsync(ws.bitmap.ptr, bitmap.data(), 4 * words, cudaMemcpyHostToDevice, st)) ||
      (T && (e = cudaMemcpyAsync(ws.tgt.ptr, tg_host.data(), 12 * (size_t)T,
                                 cudaMemcpyHostToDevice, st))) ||
      (e = cudaMemcpyAsync(ws.from.ptr, from.data(), 4 * (size_t)B, cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemsetAsync(ws.vec[0].ptr, 0, vbytes, st)) ||
      (e = cudaMemsetAsync(ws.vec[1].ptr, 0, vbytes, st)) ||
      (e = cudaMemsetAsync(ws.err.ptr, 0, 16, st)) ||
      (e = cudaMemsetAsync(ws.mu.ptr, 0, sizeof(double2) * (size_t)K * M, st)))
    return cuda_fail(e, "recursion: staging");
  if (doubling) {
    std::vector<uint32_t> col_out(Bp, kPad);
    for (uint32_t i = 0; i < T; i++) col_out[tl.col[i]] = tl.out[i];
    if ((e = cudaMemcpyAsync(ws.col_out.ptr, col_out.data(), 4 * (size_t)Bp,
                             cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemsetAsync(ws.mu_direct.ptr, 0, sizeof(double2) * (size_t)K * ld_direct, st)))
      return cuda_fail(e, "recursion: staging");
  }
  StepArgs a;
  a.A.slice_ptr = m->slice_ptr.as<uint32_t>();
  a.A.col = m->scol.as<uint32_t>();
  a.A.val = m->sval.as<double2>();
  a.A.N = m->N;
  a.A.nslices = m->nslices;
  a.A.vre = m->values_real ? m->sreal.as<double>() : nullptr;
  // FP64 head: j_0 .. j_q of every source on its ball, q common to the batch
  uint32_t q = 0;
  const uint32_t want = std::min(m->head_steps, steps >= 1 ? steps - 1 : 0u);
  if (head && doubling && is_mixed(precision) && m->pattern_symmetric && want >= 2) {
    std::vector<uint32_t> slot(B, kPad);
    for (uint32_t i = 0; i < T; i++) slot[tl.col[i]] = tl.out[i];
    if (std::find(slot.begin(), slot.end(), kPad) != slot.end())
      return fail(TBTKKPM_ERR_ARGUMENT, "recursion: a doubling source without its own target");
    std::vector<PrefixJob> jobs(B);
    for (uint32_t b = 0; b < B; b++) {
      PrefixJob &j = jobs[b];
      j.slice_ptr = a.A.slice_ptr;
      j.scol = a.A.col;
      j.sval = a.A.val;
      j.site = from[b];
      j.steps = want;
      j.M = M;
      j.ld = ld_direct;
      j.mu = ws.mu.as<double2>() + (size_t)slot[b] * M;
      j.mu_direct = ws.mu_direct.as<double2>() + (size_t)slot[b] * ld_direct;
      j.x_cur = ws.vec[0].ptr;
      j.x_prev = ws.vec[1].ptr;
      j.W = Bp;
      j.col = b;
      j.real = real ? 1u : 0u;
      j.pad = 0;
    }
    std::vector<PrefixResult> res;
    if ((rc = run_fp64_head(st, jobs, ws, res))) return rc;
    q = want;
    for (const PrefixResult &r : res) q = std::min(q, r.q);
    if (q < want) {
      // a ball outgrew the table: clear the buffers and run every source to
      // the shortest head (or start plainly when that is below 2 steps)
      if ((e = cudaMemsetAsync(ws.vec[0].ptr, 0, vbytes, st)) ||
          (e = cudaMemsetAsync(ws.vec[1].ptr, 0, vbytes, st)))
        return cuda_fail(e, "recursion: staging");
      if (q >= 2) {
        for (PrefixJob &j : jobs) j.steps = q;
        if ((rc = run_fp64_head(st, jobs, ws, res))) return rc;
      } else {
        q = 0;  // the moment rows the head touched are rewritten by the plain start
      }
    }
  }
  Targets tg;
  tg.bitmap = ws.bitmap.as<uint32_t>();
  tg.row = ws.tgt.as<uint32_t>();
  tg.col = ws.tgt.as<uint32_t>() + T;
  tg.out = ws.tgt.as<uint32_t>() + 2 * (size_t)T;
  tg.count = T;
  tg.mu = doubling ? ws.mu_direct.as<double2>() : ws.mu.as<double2>();
  tg.ld = ld_direct;
  const unsigned ib = blocks_for(std::max(B, T));
  if (q > 0) {
    // the head wrote j_q, j_{q-1} and the moments through step q
  } else if (real) {
    kpm_init_sources_real<<<ib, 256, 0, st>>>(B, Bp, ws.from.as<uint32_t>(), ws.vec[0].as<float>(),
                                              tg);
  } else if (is_mixed(precision)) {
    kpm_init_sources<float2><<<ib, 256, 0, st>>>(B, Bp, ws.from.as<uint32_t>(),
                                                ws.vec[0].as<float2>(), tg);
  } else {
    kpm_init_sources<double2><<<ib, 256, 0, st>>>(B, Bp, ws.from.as<uint32_t>(),
                                                 ws.vec[0].as<double2>(), tg);
  }
  a.Bp = Bp;
  a.tg = tg;
  a.dots = doubling ? ws.dots.as<double2>() : nullptr;
  a.err = ws.err.as<int>();
  a.plan = plan;
  a.wait_limit = m->wait_limit == TBTKKPM_WAIT_DEFAULT ? kWaitLimit : m->wait_limit;
  void *cur = ws.vec[0].ptr, *prev = ws.vec[1].ptr;
  m->timer.mark(st, 0);
  m->timer.pending = m->timer.enabled;
  m->timer.pending_steps = steps - q;
  count_launches((q > 0 ? 0 : 1) + (uint64_t)(steps - q) * (doubling ? 2 : 1));
  for (uint32_t n = q + 1; n <= steps; n++) {
    a.x = cur;
    a.y = prev;
    a.n_out = n;
    unsigned grid = 0;
    (n == 1 ? fn->first : fn->rest)(st, m->device, max_grid, a, &grid);
    if (grid == 0) return fail(TBTKKPM_ERR_UNSUPPORTED, "recursion: step %d x %d / %d not launched",
                               fn->tpr, fn->vpt, fn->minb);
    std::swap(cur, prev);
    if (doubling) {
      if (n == 1) {
        // mu_0 and mu_1 of the direct gather seed the doubling identities
        e = cudaMemcpy2DAsync(ws.mu.ptr, sizeof(double2) * M, ws.mu_direct.ptr,
                              sizeof(double2) * ld_direct, sizeof(double2) * std::min(M, 2u),
                              K, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_fail(e, "recursion: seed moments");
      }
      kpm_dots_finalize<<<Bp, kFinalizeBlock, 0, st>>>(Bp, grid, ws.dots.as<double2>(),
                                                              ws.col_out.as<uint32_t>(),
                                                              ws.mu.as<double2>(), M, M, n);
    }
  }
  if (doubling && steps == 0) {
    e = cudaMemcpy2DAsync(ws.mu.ptr, sizeof(double2) * M, ws.mu_direct.ptr,
                          sizeof(double2) * ld_direct, sizeof(double2), K,
                          cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "recursion: seed moments");
  }
  m->timer.mark(st, 1);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "recursion: launch");
  return TBTKKPM_OK;
}

// After the stream has passed a batch: a bounded device wait that ran out
// turns into TBTKKPM_ERR_TIMEOUT.
int check_device_flag(tbtkkpm_matrix *m) {
  int flag = 0;
  cudaError_t e = cudaMemcpy(&flag, m->ws.err.ptr, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "recursion: status");
  if (flag)
    return fail(TBTKKPM_ERR_TIMEOUT,
                "recursion: a bounded wait for staged rows ran out (status %d)", flag);
  return TBTKKPM_OK;
}

}  // namespace

// Damping numerators a[n] = sinh(lambda(1 - n/M)) and b = sinh(lambda),
// evaluated with the host's libm exactly as ChebyshevExpander.cpp:192-195.
void damping_factors(uint32_t M, double broadening, std::vector<double> &a, double &b) {
  const double lambda = broadening * M;
  a.resize(M);
  for (uint32_t n = 0; n < M; n++) a[n] = std::sinh(lambda * (1 - n / (double)M));
  b = std::sinh(lambda);
}

int check_precision(int precision) {
  if (precision != TBTKKPM_FP64 && precision != TBTKKPM_MIXED && precision != TBTKKPM_MIXED_DIRECT)
    return fail(TBTKKPM_ERR_ARGUMENT,
                "precision %d is none of TBTKKPM_FP64, TBTKKPM_MIXED, TBTKKPM_MIXED_DIRECT",
                precision);
  return TBTKKPM_OK;
}

// Error estimate of a doubling run for each output slot: the largest
// difference between the directly gathered moments (n <= M/2) and the
// doubling moments of the same n, relative to max |mu|, scaled by sqrt(2)
// for the moments past M/2 and by a safety factor of 4.
// Near the band edge (theta = acos|x| small) cos(n theta) stays close to 1
// for n < 1/theta, so the rounding errors of that many moments add up with
// little cancellation; their random sum grows as the square root of that
// count.  The estimate's constant was measured on 1000-point open grids,
// whose outermost node sits at theta_ref = acos(1 - 2/1001) = 0.063; a grid
// reaching closer to the edge (the Chebyshev nodes: theta = pi/(2E)) scales
// the weight by sqrt(theta_ref / theta_min), a grid that stays farther out
// keeps it.
double edge_coherence(double theta_min) {
  const double ref = std::acos(1.0 - 2.0 / 1001.0);
  return theta_min > 0 && theta_min < ref ? std::sqrt(ref / theta_min) : 1.0;
}

double grid_weight_max(const double *energies, uint32_t E, double scale) {
  double w = 0, th = M_PI;
  for (uint32_t e = 0; e < E; e++) {
    const double x = energies[e] / scale;
    w = std::max(w, 2.0 / (M_PI * scale * std::sqrt(1.0 - x * x)));
    th = std::min(th, std::acos(std::fabs(x)));
  }
  return w * edge_coherence(th);
}

// The moment estimate is an error scale of the moments the run returns; the
// energy sum multiplies a moment error by at most the grid's largest weight,
// so moment_err * wmax scales the LDOS's absolute error (measured over 600
// sampled solves of the 1000-model uneven batch against the FP64 path: the
// absolute error is at most 0.61 of it), and dividing by the result's
// largest value makes it relative, like the error it bounds.
double ldos_error_estimate(double moment_err, double wmax, const double *row, uint32_t E, bool complex) {
  double vmax = 0;
  for (uint32_t e = 0; e < E; e++)
    vmax = std::max(vmax, complex ? std::hypot(row[2 * e], row[2 * e + 1]) / M_PI : std::fabs(row[e]));
  return vmax > 0 ? moment_err * wmax / vmax : 0.0;
}

void doubling_error(const std::vector<double2> &mu, const std::vector<double2> &direct,
                    uint32_t K, uint32_t M, uint32_t ld, double *err) {
  for (uint32_t k = 0; k < K; k++) {
    double dmax = 0, scale = 0;
    for (uint32_t n = 0; n < M; n++) {
      const double2 v = mu[(size_t)k * M + n];
      scale = std::max(scale, std::hypot(v.x, v.y));
    }
    for (uint32_t n = 2; n < std::min(ld, M); n++) {
      const double2 a = mu[(size_t)k * M + n], b = direct[(size_t)k * ld + n];
      dmax = std::max(dmax, std::hypot(a.x - b.x, a.y - b.y));
    }
    err[k] = scale > 0 ? 4.0 * std::sqrt(2.0) * dmax / scale : 0.0;
  }
}

// Sources per recursion batch of a call.  A wider batch reads the matrix
// fewer times, but past a point its step slows by more than the matrix
// share it saves.  Doubling steps per source and step: real float vectors
// on the 2048^2 lattice 0.0385 ms at 128 sources against 0.0465 ms at 256;
// complex64 vectors on the 1024^2 Rashba lattice 0.0261 ms at 128 against
// 0.0327 ms at 256 (0.0303 at 64).  So doubling runs split at 128.
uint32_t batch_width_for(const tbtkkpm_matrix *m, int precision, bool doubling) {
  const uint32_t maxb = is_mixed(precision) ? kMaxBatchMixed : kMaxBatchFP64;
  const uint32_t set = m->batch_width[precision];
  if (set) return std::min(set, maxb);
  if (doubling) return 128;
  return maxb;
}

// Moments of several batches: sources split into batches of at most
// batch_width_for sources; to-indices follow their owner.  Results land in host
// memory mu_out ([K][M]) undamped.
static int moments_host(tbtkkpm_matrix *m, const uint32_t *from, uint32_t B, const uint32_t *to,
                        const uint32_t *owner, uint32_t K, uint32_t M, int precision,
                        double *mu_out) {
  const uint32_t maxb = batch_width_for(m, precision, false);
  std::vector<std::vector<uint32_t>> by_owner(B);
  for (uint32_t k = 0; k < K; k++) by_owner[owner[k]].push_back(k);
  std::vector<double2> mu_host;
  for (uint32_t b0 = 0; b0 < B; b0 += maxb) {
    const uint32_t nb = std::min(maxb, B - b0);
    std::vector<uint32_t> fr(from + b0, from + b0 + nb);
    std::vector<std::array<uint32_t, 3>> items;  // row, column, output slot (local)
    std::vector<uint32_t> global_k;
    for (uint32_t b = 0; b < nb; b++)
      for (uint32_t k : by_owner[b0 + b]) {
        items.push_back({to[k], b, (uint32_t)global_k.size()});
        global_k.push_back(k);
      }
    if (items.empty()) continue;
    std::stable_sort(items.begin(), items.end(),
                     [](const std::array<uint32_t, 3> &a, const std::array<uint32_t, 3> &b) {
                       return a[0] < b[0];
                     });
    TargetList tl;
    for (auto &it : items) {
      tl.row.push_back(it[0]);
      tl.col.push_back(it[1]);
      tl.out.push_back(it[2]);
    }
    const uint32_t Kb = (uint32_t)global_k.size();
    int rc = run_batch(m, precision, fr, tl, Kb, M, false);
    if (rc) return rc;
    mu_host.resize((size_t)Kb * M);
    m->timer.mark(m->stream, 2);
    m->timer.mark(m->stream, 3);
    cudaError_t e = cudaMemcpyAsync(mu_host.data(), m->ws.mu.ptr, sizeof(double2) * Kb * M,
                                    cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    if (e != cudaSuccess) return cuda_fail(e, "moments: download");
    m->timer.collect();
    if ((rc = check_device_flag(m))) return rc;
    for (uint32_t i = 0; i < Kb; i++)
      std::memcpy(mu_out + 2 * (size_t)global_k[i] * M, mu_host.data() + (size_t)i * M,
                  sizeof(double2) * M);
  }
  return TBTKKPM_OK;
}

// Lorentz damping on the host, c*a/b component-wise
// (ChebyshevExpander.cpp:190-196).
static void damp_host(uint32_t K, uint32_t M, double broadening, double *mu) {
  if (broadening == 0) return;
  std::vector<double> a;
  double b;
  damping_factors(M, broadening, a, b);
  for (uint32_t k = 0; k < K; k++)
    for (uint32_t n = 0; n < M; n++) {
      double *c = mu + 2 * ((size_t)k * M + n);
      c[0] = c[0] * a[n] / b;
      c[1] = c[1] * a[n] / b;
    }
}

static int check_moment_args(tbtkkpm_matrix *m, const uint32_t *from, uint32_t B,
                             const uint32_t *to, const uint32_t *owner, uint32_t K, uint32_t M,
                             double broadening, double *mu_out, const char *fn) {
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "%s: NULL matrix", fn);
  if (M == 0) return fail(TBTKKPM_ERR_ARGUMENT, "%s: numCoefficients has to be larger than 0", fn);
  if (B == 0 || !from) return fail(TBTKKPM_ERR_ARGUMENT, "%s: no source index", fn);
  if (K && (!to || !mu_out)) return fail(TBTKKPM_ERR_ARGUMENT, "%s: NULL to/mu_out", fn);
  if (!std::isfinite(broadening)) return fail(TBTKKPM_ERR_ARGUMENT, "%s: broadening not finite", fn);
  for (uint32_t b = 0; b < B; b++)
    if (from[b] >= m->N)
      return fail(TBTKKPM_ERR_ARGUMENT, "%s: from index %u outside the basis of size %u", fn,
                  from[b], m->N);
  for (uint32_t k = 0; k < K; k++) {
    if (to[k] >= m->N)
      return fail(TBTKKPM_ERR_ARGUMENT, "%s: to index %u outside the basis of size %u", fn,
                  to[k], m->N);
    if (owner && owner[k] >= B)
      return fail(TBTKKPM_ERR_ARGUMENT, "%s: to_owner[%u]=%u >= B=%u", fn, k, owner[k], B);
  }
  return TBTKKPM_OK;
}

}  // namespace tbtkkpm

using namespace tbtkkpm;

extern "C" int tbtkkpm_moments(tbtkkpm_matrix *m, uint32_t from, const uint32_t *to, uint32_t K,
                               uint32_t M, double broadening, double *mu_out) {
  int rc = check_moment_args(m, &from, 1, to, nullptr, K, M, broadening, mu_out, "moments");
  if (rc) return rc;
  if (K == 0) return TBTKKPM_OK;
  std::lock_guard<std::mutex> lk(m->lock);
  DeviceGuard g(m->device);
  std::vector<uint32_t> owner(K, 0u);
  rc = moments_host(m, &from, 1, to, owner.data(), K, M, TBTKKPM_FP64, mu_out);
  if (rc) return rc;
  damp_host(K, M, broadening, mu_out);
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_moments_batched(tbtkkpm_matrix *m, const uint32_t *from, uint32_t B,
                                       const uint32_t *to, const uint32_t *to_owner, uint32_t K,
                                       uint32_t M, double broadening, int precision,
                                       double *mu_out, double *err_out) {
  int rc = check_precision(precision);
  if (rc) return rc;
  if (K && !to_owner) return fail(TBTKKPM_ERR_ARGUMENT, "moments_batched: NULL to_owner");
  rc = check_moment_args(m, from, B, to, to_owner, K, M, broadening, mu_out, "moments_batched");
  if (rc) return rc;
  if (K == 0) return TBTKKPM_OK;
  std::lock_guard<std::mutex> lk(m->lock);
  DeviceGuard g(m->device);
  rc = moments_host(m, from, B, to, to_owner, K, M, precision, mu_out);
  if (rc) return rc;
  damp_host(K, M, broadening, mu_out);
  if (err_out)
    for (uint32_t k = 0; k < K; k++) err_out[k] = is_mixed(precision) ? -1.0 : 0.0;
  return TBTKKPM_OK;
}

// ---------------------------------------------------------------- tables

static int table_alloc(uint32_t M, uint32_t E, tbtkkpm_table **out, bool with_table = true) {
  int ndev = 0;
  tbtkkpm_device_count(&ndev);
  if (ndev == 0) return fail(TBTKKPM_ERR_CUDA, "no CUDA device available");
  auto *t = new tbtkkpm_table();
  t->device = current_device();
  t->M = M;
  t->E = E;
  DeviceGuard g(t->device);
  cudaError_t e = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete t;
    return cuda_fail(e, "cudaStreamCreate");
  }
  int rc = with_table ? t->table.reserve(sizeof(double2) * (size_t)M * E) : TBTKKPM_OK;
  if (rc) {
    tbtkkpm_table_destroy(t);
    return rc;
  }
  *out = t;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_table_create(uint32_t M, const double *energies, uint32_t E, double scale,
                                    tbtkkpm_table **out) {
  if (!out) return fail(TBTKKPM_ERR_ARGUMENT, "table_create: out is NULL");
  *out = nullptr;
  if (M == 0) return fail(TBTKKPM_ERR_ARGUMENT, "table_create: numCoefficients has to be larger than 0");
  if (E == 0 || !energies)
    return fail(TBTKKPM_ERR_ARGUMENT, "table_create: The energy windows resolution has to be larger than 0.");
  if (!(scale > 0)) return fail(TBTKKPM_ERR_ARGUMENT, "table_create: scaleFactor must be > 0");
  for (uint32_t e = 0; e < E; e++)
    if (!(energies[e] > -scale && energies[e] < scale))
      return fail(TBTKKPM_ERR_ARGUMENT,
                  "table_create: energy %g is not contained in the interval (-scaleFactor, "
                  "scaleFactor)=(%g, %g)",
                  energies[e], -scale, scale);
  tbtkkpm_table *t = nullptr;
  int rc = table_alloc(M, E, &t);
  if (rc) return rc;
  t->wmax = grid_weight_max(energies, E, scale);
  DeviceGuard g(t->device);
  DevBuf en;
  if ((rc = en.reserve(8 * (size_t)E))) {
    tbtkkpm_table_destroy(t);
    return rc;
  }
  cudaMemcpyAsync(en.ptr, energies, 8 * (size_t)E, cudaMemcpyHostToDevice, t->stream);
  kpm_table_gen<<<blocks_for((uint64_t)M * E), 256, 0, t->stream>>>(M, E, en.as<double>(), scale,
                                                                     t->table.as<double2>());
  count_launches(1);
  cudaError_t e = cudaStreamSynchronize(t->stream);
  en.release();
  if (e != cudaSuccess) {
    tbtkkpm_table_destroy(t);
    return cuda_fail(e, "table_create");
  }
  *out = t;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_table_create_clenshaw(uint32_t M, const double *energies, uint32_t E,
                                             double scale, tbtkkpm_table **out) {
  if (!out) return fail(TBTKKPM_ERR_ARGUMENT, "table_create_clenshaw: out is NULL");
  *out = nullptr;
  if (M == 0)
    return fail(TBTKKPM_ERR_ARGUMENT, "table_create_clenshaw: numCoefficients has to be larger than 0");
  if (E == 0 || !energies)
    return fail(TBTKKPM_ERR_ARGUMENT,
                "table_create_clenshaw: The energy windows resolution has to be larger than 0.");
  if (!(scale > 0)) return fail(TBTKKPM_ERR_ARGUMENT, "table_create_clenshaw: scaleFactor must be > 0");
  for (uint32_t e = 0; e < E; e++)
    if (!(energies[e] > -scale && energies[e] < scale))
      return fail(TBTKKPM_ERR_ARGUMENT,
                  "table_create_clenshaw: energy %g is not contained in the interval (-scaleFactor, "
                  "scaleFactor)=(%g, %g)",
                  energies[e], -scale, scale);
  tbtkkpm_table *t = nullptr;
  int rc = table_alloc(M, E, &t, false);
  if (rc) return rc;
  DeviceGuard g(t->device);
  t->clenshaw = true;
  t->scale = scale;
  t->wmax = grid_weight_max(energies, E, scale);
  if ((rc = t->energies.reserve(8 * (size_t)E))) {
    tbtkkpm_table_destroy(t);
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(t->energies.ptr, energies, 8 * (size_t)E, cudaMemcpyHostToDevice,
                                  t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  if (e != cudaSuccess) {
    tbtkkpm_table_destroy(t);
    return cuda_fail(e, "table_create_clenshaw");
  }
  *out = t;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_table_create_chebyshev(uint32_t M, uint32_t E, double scale,
                                              double *energies_out, tbtkkpm_table **out) {
  if (!out) return fail(TBTKKPM_ERR_ARGUMENT, "table_create_chebyshev: out is NULL");
  *out = nullptr;
  if (M == 0)
    return fail(TBTKKPM_ERR_ARGUMENT, "table_create_chebyshev: numCoefficients has to be larger than 0");
  if (E == 0 || (E & (E - 1)) || E > kDctMaxE)
    return fail(TBTKKPM_ERR_ARGUMENT,
                "table_create_chebyshev: the number of energies (%u) has to be a power of two in "
                "[1, %u]",
                E, kDctMaxE);
  if (!(scale > 0)) return fail(TBTKKPM_ERR_ARGUMENT, "table_create_chebyshev: scaleFactor must be > 0");
  if (!energies_out) return fail(TBTKKPM_ERR_ARGUMENT, "table_create_chebyshev: energies_out is NULL");
  const uint32_t L = 2 * E;
  std::vector<double2> tw(L);
  for (uint32_t m = 0; m < L; m++) {
    const double a = M_PI * (double)m / (double)L;
    tw[m] = make_double2(std::cos(a), std::sin(a));
  }
  // node k = E - 1 - e at x_k = cos(pi (2k + 1) / L): ascending energies
  std::vector<double> en(E);
  for (uint32_t e = 0; e < E; e++) en[e] = scale * tw[2 * (E - 1 - e) + 1].x;
  tbtkkpm_table *t = nullptr;
  int rc = table_alloc(M, E, &t, false);
  if (rc) return rc;
  DeviceGuard g(t->device);
  t->chebyshev_grid = true;
  t->scale = scale;
  t->wmax = grid_weight_max(en.data(), E, scale);
  if ((rc = t->twiddle.reserve(sizeof(double2) * (size_t)L))) {
    tbtkkpm_table_destroy(t);
    return rc;
  }
  cudaError_t e = cudaMemcpyAsync(t->twiddle.ptr, tw.data(), sizeof(double2) * (size_t)L,
                                  cudaMemcpyHostToDevice, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  if (e != cudaSuccess) {
    tbtkkpm_table_destroy(t);
    return cuda_fail(e, "table_create_chebyshev");
  }
  std::copy(en.begin(), en.end(), energies_out);
  *out = t;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_table_upload(uint32_t M, uint32_t E, const double *table,
                                    tbtkkpm_table **out) {
  if (!out) return fail(TBTKKPM_ERR_ARGUMENT, "table_upload: out is NULL");
  *out = nullptr;
  if (M == 0 || E == 0 || !table) return fail(TBTKKPM_ERR_ARGUMENT, "table_upload: empty table");
  tbtkkpm_table *t = nullptr;
  int rc = table_alloc(M, E, &t);
  if (rc) return rc;
  // |T[1][e]| = 2 / (s sqrt(1 - x^2)); T[0][e] carries half of it.
  // T[1][e] = (2/(s q)) e^{-i(theta + pi/2)} gives the node's angle theta
  double th = M_PI;
  for (uint32_t e = 0; e < E; e++) {
    const double *v = table + 2 * ((size_t)(M > 1 ? E : 0) + e);
    t->wmax = std::max(t->wmax, (M > 1 ? 1.0 : 2.0) * std::hypot(v[0], v[1]) / M_PI);
    if (M > 1) {
      double a = std::remainder(-std::atan2(v[1], v[0]) - M_PI / 2, 2 * M_PI);  // theta in [0, pi]
      a = std::fabs(a);
      th = std::min(th, std::min(a, M_PI - a));
    }
  }
  t->wmax *= edge_coherence(th);
  DeviceGuard g(t->device);
  cudaError_t e = cudaMemcpyAsync(t->table.ptr, table, sizeof(double2) * (size_t)M * E,
                                  cudaMemcpyHostToDevice, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  if (e != cudaSuccess) {
    tbtkkpm_table_destroy(t);
    return cuda_fail(e, "table_upload");
  }
  *out = t;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_table_destroy(tbtkkpm_table *t) {
  if (!t) return TBTKKPM_OK;
  {
    DeviceGuard g(t->device);
    if (t->stream) cudaStreamSynchronize(t->stream);
    t->table.release();
    t->energies.release();
    t->twiddle.release();
    t->mu.release();
    t->out.release();
    if (t->stream) cudaStreamDestroy(t->stream);
  }
  delete t;
  return TBTKKPM_OK;
}

namespace tbtkkpm {

// Launches the energy sum of `type` (0-3 Green's functions, 4 = LDOS) for K
// coefficient vectors resident on the device ([K][M] with M = terms, or the
// table's M when terms is 0; a table of more rows serves fewer terms).
int launch_energy_sum(cudaStream_t st, const tbtkkpm_table *t, const double2 *mu, uint32_t K,
                      int type, void *out, uint32_t terms) {
  const uint32_t M = terms ? terms : t->M, E = t->E;
  if (K == 0) return TBTKKPM_OK;
  if (t->chebyshev_grid) {
    uint32_t log2L = 0;
    while ((1u << log2L) < 2 * E) log2L++;
    const int smem = (int)(sizeof(double2) * 2 * E);
    cudaError_t e = cudaSuccess;
    if (smem > 48 * 1024)
      e = cudaFuncSetAttribute(kpm_chebyshev_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return cuda_fail(e, "energy sum: shared memory");
    kpm_chebyshev_grid<<<K, kDctBlock, smem, st>>>(M, E, log2L, t->twiddle.as<double2>(), t->scale,
                                                    mu, type, out);
    count_launches(1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "energy sum: launch");
    return TBTKKPM_OK;
  }
  const int KT = K == 1 ? 1 : (K <= 4 ? 4 : 8);
  dim3 grid((E + kEnergyBlock - 1) / kEnergyBlock, (K + KT - 1) / KT);
  if (t->clenshaw) {
    const double *en = t->energies.as<double>();
    if (KT == 1)
      kpm_clenshaw<1><<<grid, kEnergyBlock, 0, st>>>(M, E, K, en, t->scale, mu, type, out);
    else if (KT == 4)
      kpm_clenshaw<4><<<grid, kEnergyBlock, 0, st>>>(M, E, K, en, t->scale, mu, type, out);
    else
      kpm_clenshaw<8><<<grid, kEnergyBlock, 0, st>>>(M, E, K, en, t->scale, mu, type, out);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "energy sum: launch");
    return TBTKKPM_OK;
  }
  const double2 *tb = t->table.as<double2>();
#define TBTKKPM_G(TY, KK) \
  kpm_greens<TY, KK><<<grid, kEnergyBlock, 0, st>>>(M, E, K, tb, mu, static_cast<double2 *>(out))
#define TBTKKPM_TYPES(KK)                       \
  switch (type) {                               \
    case 0: TBTKKPM_G(0, KK); break;            \
    case 1: TBTKKPM_G(1, KK); break;            \
    case 2: TBTKKPM_G(2, KK); break;            \
    case 3: TBTKKPM_G(3, KK); break;            \
    default:                                    \
      kpm_ldos<KK><<<grid, kEnergyBlock, 0, st>>>(M, E, K, tb, mu, static_cast<double *>(out)); \
  }
  if (KT == 1) {
    TBTKKPM_TYPES(1)
  } else if (KT == 4) {
    TBTKKPM_TYPES(4)
  } else {
    TBTKKPM_TYPES(8)
  }
#undef TBTKKPM_TYPES
#undef TBTKKPM_G
  count_launches(1);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "energy sum: launch");
  return TBTKKPM_OK;
}

// Energy sum of host moments [K][terms] (terms 0: the table's M; a table of
// more rows serves fewer terms with the same sums) into host `out`.
int energy_sum_host(tbtkkpm_table *t, const double *mu, uint32_t K, int type, void *out,
                    size_t out_elem, uint32_t terms) {
  std::lock_guard<std::mutex> lk(t->lock);
  DeviceGuard g(t->device);
  const uint32_t M = terms ? terms : t->M;
  const size_t mbytes = sizeof(double2) * (size_t)K * M;
  const size_t obytes = out_elem * (size_t)K * t->E;
  int rc;
  if ((rc = t->mu.reserve(mbytes)) || (rc = t->out.reserve(obytes))) return rc;
  cudaError_t e = cudaMemcpyAsync(t->mu.ptr, mu, mbytes, cudaMemcpyHostToDevice, t->stream);
  if (e != cudaSuccess) return cuda_fail(e, "energy sum: upload");
  if ((rc = launch_energy_sum(t->stream, t, t->mu.as<double2>(), K, type, t->out.ptr, M))) return rc;
  e = cudaMemcpyAsync(out, t->out.ptr, obytes, cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  if (e != cudaSuccess) return cuda_fail(e, "energy sum: download");
  return TBTKKPM_OK;
}

}  // namespace tbtkkpm

extern "C" int tbtkkpm_greens(tbtkkpm_table *t, const double *mu, uint32_t K, int type,
                              double *G_out) {
  if (!t) return fail(TBTKKPM_ERR_ARGUMENT, "greens: NULL table");
  if (type < 0 || type > 3) return fail(TBTKKPM_ERR_ARGUMENT, "greens: Unkown Green's function type %d", type);
  if (K == 0) return TBTKKPM_OK;
  if (!mu || !G_out) return fail(TBTKKPM_ERR_ARGUMENT, "greens: NULL buffers");
  return energy_sum_host(t, mu, K, type, G_out, sizeof(double2), 0);
}

extern "C" int tbtkkpm_ldos(tbtkkpm_table *t, const double *mu, uint32_t K, double *ldos_out) {
  if (!t) return fail(TBTKKPM_ERR_ARGUMENT, "ldos: NULL table");
  if (K == 0) return TBTKKPM_OK;
  if (!mu || !ldos_out) return fail(TBTKKPM_ERR_ARGUMENT, "ldos: NULL buffers");
  return energy_sum_host(t, mu, K, 4, ldos_out, sizeof(double), 0);
}

extern "C" int tbtkkpm_ldos_sites(tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *sites,
                                  uint32_t B, double broadening, int precision, double *ldos_out,
                                  double *err_out) {
  if (!t) return fail(TBTKKPM_ERR_ARGUMENT, "ldos_sites: NULL table");
  return tbtkkpm::ldos_sites_terms(m, t, t->M, sites, B, broadening, precision, ldos_out, err_out);
}

// tbtkkpm_ldos_sites with M <= the table's rows moments: a table of more
// rows gives the same sums as one of M rows.
int tbtkkpm::ldos_sites_terms(tbtkkpm_matrix *m, tbtkkpm_table *t, uint32_t M, const uint32_t *sites,
                              uint32_t B, double broadening, int precision, double *ldos_out,
                              double *err_out) {
  int rc = check_precision(precision);
  if (rc) return rc;
  if (!t) return fail(TBTKKPM_ERR_ARGUMENT, "ldos_sites: NULL table");
  if (B && !ldos_out) return fail(TBTKKPM_ERR_ARGUMENT, "ldos_sites: NULL ldos_out");
  if (M == 0 || M > t->M) return fail(TBTKKPM_ERR_ARGUMENT, "ldos_sites: %u moments for a table of %u", M, t->M);
  const uint32_t E = t->E;
  if (B == 0) return TBTKKPM_OK;
  rc = check_moment_args(m, sites, B, sites, nullptr, B, M, broadening, ldos_out, "ldos_sites");
  if (rc) return rc;
  if (m->device != t->device)
    return fail(TBTKKPM_ERR_ARGUMENT, "ldos_sites: matrix and table live on different devices");
  std::lock_guard<std::mutex> lk(m->lock);
  DeviceGuard g(m->device);
  const bool doubling = precision == TBTKKPM_MIXED;
  const uint32_t maxb = batch_width_for(m, precision, doubling);
  std::vector<double> a;
  double b = 1;
  const bool damp = broadening != 0;
  if (damp) damping_factors(M, broadening, a, b);
  Workspace &ws = m->ws;
  if ((rc = ws.damp.reserve(8 * (size_t)M)) ||
      (rc = ws.out.reserve(sizeof(double) * (size_t)std::min(B, maxb) * E)))
    return rc;
  cudaError_t e;
  if (damp && (e = cudaMemcpyAsync(ws.damp.ptr, a.data(), 8 * (size_t)M, cudaMemcpyHostToDevice,
                                   m->stream)) != cudaSuccess)
    return cuda_fail(e, "ldos_sites: damping upload");
  // Table reads happen on the matrix stream; order them after the table's own work.
  cudaStreamSynchronize(t->stream);
  std::vector<double2> mu_h, direct_h;
  for (uint32_t b0 = 0; b0 < B; b0 += maxb) {
    const uint32_t nb = std::min(maxb, B - b0);
    std::vector<uint32_t> fr(sites + b0, sites + b0 + nb);
    std::vector<std::array<uint32_t, 2>> items;
    for (uint32_t i = 0; i < nb; i++) items.push_back({fr[i], i});
    std::stable_sort(items.begin(), items.end(),
                     [](const std::array<uint32_t, 2> &x, const std::array<uint32_t, 2> &y) {
                       return x[0] < y[0];
                     });
    TargetList tl;
    for (auto &it : items) {
      tl.row.push_back(it[0]);
      tl.col.push_back(it[1]);
      tl.out.push_back(it[1]);
    }
    if ((rc = run_batch(m, precision, fr, tl, nb, M, doubling))) return rc;
    const uint32_t ld = M / 2 + 1;
    if (doubling && err_out) {
      // undamped moments for the estimate
      mu_h.resize((size_t)nb * M);
      direct_h.resize((size_t)nb * ld);
      cudaMemcpyAsync(mu_h.data(), ws.mu.ptr, sizeof(double2) * nb * M, cudaMemcpyDeviceToHost,
                      m->stream);
      cudaMemcpyAsync(direct_h.data(), ws.mu_direct.ptr, sizeof(double2) * nb * ld,
                      cudaMemcpyDeviceToHost, m->stream);
    }
    if (doubling) {
      // Moments n <= M/2 were gathered directly as well; those carry less
      // rounding than the dot-product identities, so they replace the
      // doubled values, which remain only past M/2 where the damping
      // sinh(lambda(1-n/M))/sinh(lambda) shrinks their weight.
      e = cudaMemcpy2DAsync(ws.mu.ptr, sizeof(double2) * M, ws.mu_direct.ptr,
                            sizeof(double2) * ld, sizeof(double2) * std::min(ld, M), nb,
                            cudaMemcpyDeviceToDevice, m->stream);
      if (e != cudaSuccess) return cuda_fail(e, "ldos_sites: direct moments");
    }
    m->timer.mark(m->stream, 2);
    if (damp) {
      kpm_damp<<<blocks_for((uint64_t)nb * M), 256, 0, m->stream>>>(nb, M, ws.damp.as<double>(), b,
                                                                   ws.mu.as<double2>());
      count_launches(1);
    }
    if ((rc = launch_energy_sum(m->stream, t, ws.mu.as<double2>(), nb, 4, ws.out.ptr, M))) return rc;
    m->timer.mark(m->stream, 3);
    e = cudaMemcpyAsync(ldos_out + (size_t)b0 * E, ws.out.ptr, sizeof(double) * (size_t)nb * E,
                        cudaMemcpyDeviceToHost, m->stream);
    if (e != cudaSuccess) return cuda_fail(e, "ldos_sites: download");
    // one synchronisation per batch of up to 256 sites (seconds of work at
    // full size): timers, the error estimate and the device status
    if ((e = cudaStreamSynchronize(m->stream)) != cudaSuccess) return cuda_fail(e, "ldos_sites");
    m->timer.collect();
    if ((rc = check_device_flag(m))) return rc;
    if (err_out) {
      if (doubling) {
        doubling_error(mu_h, direct_h, nb, M, ld, err_out + b0);
        for (uint32_t i = 0; i < nb; i++)
          err_out[b0 + i] = ldos_error_estimate(err_out[b0 + i], t->wmax,
                                                ldos_out + (size_t)(b0 + i) * E, E, false);
      } else
        for (uint32_t i = 0; i < nb; i++) err_out[b0 + i] = is_mixed(precision) ? -1.0 : 0.0;
    }
  }
  if ((e = cudaStreamSynchronize(m->stream)) != cudaSuccess) return cuda_fail(e, "ldos_sites");
  return TBTKKPM_OK;
}

// ---------------------------------------------------------------- autotuner
// Times every compiled step configuration whose padded width serves B
// sources on this matrix (probe_steps steps each, best of two runs, CUDA
// events on the handle's stream around the steps) and keeps the fastest for
// later batches of that width on this handle.
extern "C" int tbtkkpm_matrix_autotune(tbtkkpm_matrix *m, uint32_t B, int precision, int ldos,
                                       uint32_t probe_steps, int *tpr, int *vpt, int *minb,
                                       double *ms_per_step) {
  int rc = check_precision(precision);
  if (rc) return rc;
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_autotune: NULL matrix");
  const uint32_t maxb = is_mixed(precision) ? kMaxBatchMixed : kMaxBatchFP64;
  if (B == 0 || B > maxb || B > m->N)
    return fail(TBTKKPM_ERR_ARGUMENT, "matrix_autotune: batch %u outside [1, %u]", B,
                std::min(maxb, m->N));
  if (probe_steps == 0) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_autotune: probe_steps is 0");
  std::lock_guard<std::mutex> lk(m->lock);
  DeviceGuard g(m->device);
  const bool doubling = ldos && precision == TBTKKPM_MIXED;
  const bool real = real_mode(m, precision);
  const int cls = step_class(precision, doubling, real);
  const uint32_t Bp = shape_for(precision, B, real).bp();
  const uint32_t M = doubling ? 2 * probe_steps : probe_steps + 1;
  std::vector<uint32_t> fr(B);
  for (uint32_t b = 0; b < B; b++) fr[b] = (uint32_t)((uint64_t)b * m->N / B);
  TargetList tl;
  for (uint32_t b = 0; b < B; b++) {
    tl.row.push_back(fr[b]);
    tl.col.push_back(b);
    tl.out.push_back(b);
  }
  PhaseTimer saved = m->timer;
  if ((rc = m->timer.enable(true))) return rc;
  const StepEntry *t;
  int n;
  step_table(cls, &t, &n);
  const StepEntry *best = nullptr;
  double best_ms = 0;
  for (int i = 0; i < n; i++) {
    if ((uint32_t)(t[i].tpr * t[i].vpt) != Bp) continue;
    double ms = 0;
    bool skip = false;
    for (int rep = 0; rep < 2; rep++) {
      m->timer.recursion_ms = 0;
      if ((rc = run_batch(m, precision, fr, tl, B, M, doubling, &t[i], false))) {
        // a tile-staged step whose ring does not fit this matrix
        if (rc == TBTKKPM_ERR_UNSUPPORTED && is_tiled_variant(t[i].minb)) {
          rc = TBTKKPM_OK;
          skip = true;
        }
        break;
      }
      cudaError_t e = cudaStreamSynchronize(m->stream);
      if (e != cudaSuccess) {
        rc = cuda_fail(e, "matrix_autotune");
        break;
      }
      m->timer.collect();
      if ((rc = check_device_flag(m))) break;
      const double v = m->timer.recursion_ms / probe_steps;
      ms = rep == 0 ? v : std::min(ms, v);
    }
    if (rc) break;
    if (skip) continue;
    if (!best || ms < best_ms) {
      best = &t[i];
      best_ms = ms;
    }
  }
  const bool created = saved.ev[0] == nullptr;
  if (created) m->timer.destroy();
  else {
    m->timer.enabled = saved.enabled;
    m->timer.recursion_ms = saved.recursion_ms;
    m->timer.energy_ms = saved.energy_ms;
    m->timer.step_launches = saved.step_launches;
    m->timer.pending = false;
  }
  if (rc) return rc;
  if (!best) return fail(TBTKKPM_ERR_UNSUPPORTED, "matrix_autotune: no configuration for %u", B);
  m->tuned[tune_key(cls, Bp)] = {best->tpr, best->vpt, best->minb};
  {
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    g_tuned[shape_key(m, cls, Bp)] = {best->tpr, best->vpt, best->minb};
  }
  if (tpr) *tpr = best->tpr;
  if (vpt) *vpt = best->vpt;
  if (minb) *minb = best->minb;
  if (ms_per_step) *ms_per_step = best_ms;
  return TBTKKPM_OK;
}

// Records a configuration for batches of B sources without timing (a
// cached autotuner result).
extern "C" int tbtkkpm_matrix_set_config(tbtkkpm_matrix *m, uint32_t B, int precision, int ldos,
                                         int tpr, int vpt, int minb) {
  int rc = check_precision(precision);
  if (rc) return rc;
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_set_config: NULL matrix");
  const bool doubling = ldos && precision == TBTKKPM_MIXED;
  const bool real = real_mode(m, precision);
  const int cls = step_class(precision, doubling, real);
  const uint32_t Bp = shape_for(precision, std::max(B, 1u), real).bp();
  if ((uint32_t)(tpr * vpt) != Bp || !find_step(cls, tpr, vpt, minb))
    return fail(TBTKKPM_ERR_ARGUMENT, "matrix_set_config: no compiled configuration %d x %d / %d "
                "for %u columns", tpr, vpt, minb, Bp);
  std::lock_guard<std::mutex> lk(m->lock);
  m->tuned[tune_key(cls, Bp)] = {tpr, vpt, minb};
  return TBTKKPM_OK;
}

// The compiled step configurations of the kernel class a call at this
// precision uses (ldos != 0: tbtkkpm_ldos_sites), as (tpr, vpt, variant)
// triples; returns how many there are (writes at most cap triples).
extern "C" int tbtkkpm_step_configs(int precision, int ldos, int *out, int cap) {
  if (check_precision(precision)) return -1;
  const StepEntry *t;
  int n;
  step_table(step_class(precision, ldos && precision == TBTKKPM_MIXED), &t, &n);
  for (int i = 0; i < n && i < cap && out; i++) {
    out[3 * i] = t[i].tpr;
    out[3 * i + 1] = t[i].vpt;
    out[3 * i + 2] = t[i].minb;
  }
  return n;
}

// As tbtkkpm_step_configs for the kernels this matrix uses (real-vector
// kernels for a real matrix at mixed precision).
extern "C" int tbtkkpm_matrix_step_configs(tbtkkpm_matrix *m, int precision, int ldos, int *out,
                                           int cap) {
  if (!m || check_precision(precision)) return -1;
  const StepEntry *t;
  int n;
  step_table(step_class(precision, ldos && precision == TBTKKPM_MIXED, real_mode(m, precision)),
             &t, &n);
  for (int i = 0; i < n && i < cap && out; i++) {
    out[3 * i] = t[i].tpr;
    out[3 * i + 1] = t[i].vpt;
    out[3 * i + 2] = t[i].minb;
  }
  return n;
}

extern "C" int tbtkkpm_matrix_set_real(tbtkkpm_matrix *m, int enable) {
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_set_real: NULL matrix");
  std::lock_guard<std::mutex> lk(m->lock);
  m->use_real = enable != 0;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_set_fp64_head(tbtkkpm_matrix *m, uint32_t steps) {
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_set_fp64_head: NULL matrix");
  std::lock_guard<std::mutex> lk(m->lock);
  m->head_steps = steps;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_set_wait_limit(tbtkkpm_matrix *m, uint32_t polls) {
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_set_wait_limit: NULL matrix");
  std::lock_guard<std::mutex> lk(m->lock);
  m->wait_limit = polls;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_fp64_head(tbtkkpm_matrix *m, uint32_t *steps, int *pattern_symmetric) {
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_fp64_head: NULL matrix");
  if (steps) *steps = m->head_steps;
  if (pattern_symmetric) *pattern_symmetric = m->pattern_symmetric ? 1 : 0;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_set_batch_width(tbtkkpm_matrix *m, int precision,
                                              uint32_t width) {
  int rc = check_precision(precision);
  if (rc) return rc;
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_set_batch_width: NULL matrix");
  const uint32_t maxb = is_mixed(precision) ? kMaxBatchMixed : kMaxBatchFP64;
  if (width > maxb)
    return fail(TBTKKPM_ERR_ARGUMENT, "matrix_set_batch_width: %u sources above the maximum %u",
                width, maxb);
  std::lock_guard<std::mutex> lk(m->lock);
  m->batch_width[precision] = width;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_batch_width(tbtkkpm_matrix *m, int precision, int ldos,
                                          uint32_t *width) {
  int rc = check_precision(precision);
  if (rc) return rc;
  if (!m || !width) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_batch_width: NULL argument");
  std::lock_guard<std::mutex> lk(m->lock);
  *width = batch_width_for(m, precision, ldos && precision == TBTKKPM_MIXED);
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_real(tbtkkpm_matrix *m, int *values_real, int *in_use) {
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_real: NULL matrix");
  if (values_real) *values_real = m->values_real ? 1 : 0;
  if (in_use) *in_use = (m->values_real && m->use_real) ? 1 : 0;
  return TBTKKPM_OK;
}
