// The server behind tbtkkpm_server_* (include/tbtkkpm.h): continuous
// batching of LDOS and Green's-function requests over many device-resident
// models.
//
// One worker thread per server repeats
//   admit  - queued requests take free lanes of their model (one per
//            source) at the next step boundary; a model's lane memory is
//            allocated on its first request within the HBM budget, evicting
//            idle models (LRU);
//   tick   - joins (column = e_source, or an FP64 head), then S steps of
//            every lane class (width, real or complex lanes) over all
//            models with busy lanes, S ending no later than the first lane
//            that finishes: one step of every class captured as a CUDA
//            graph and replayed S times, the classes on their own streams;
//   finish - for every finished request: moments damped and summed over the
//            energy grid on the device (LDOS or the request's Green's
//            function type), the error estimate, release of the lanes.
// A second thread runs the FP64 recomputations of outputs past the
// tolerance, so the worker keeps stepping meanwhile.  Submitters only queue
// and wait.
#include "tbtkkpm.h"
#include "kpm_host.h"
#include "kpm_multi.cuh"
#include "kpm_multi_real.cuh"
#include "kpm_multi_tiled.cuh"
#include "kpm_prefix.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

namespace tbtkkpm {
namespace {

using Clock = std::chrono::steady_clock;

inline unsigned blocks_for(uint64_t n, unsigned bs = 256) { return (unsigned)((n + bs - 1) / bs); }

constexpr uint32_t kMaxWidth = 64;

bool valid_width(uint32_t w) { return w >= 1 && w <= kMaxWidth && (w & (w - 1)) == 0; }

constexpr int kLdos = -1;  // Request::kind of an LDOS request

// Narrowest width a model steps at when its width follows demand: below it
// the matrix bytes of a step dominate and a narrower row saves little.
constexpr uint32_t kMinStepWidth = 4;

struct Request {
  uint64_t id = 0;
  uint32_t model = 0;
  int kind = kLdos;  // kLdos, or the Green's function type (TBTKKPM_ADVANCED..NONPRINCIPAL)
  // the sources, one lane each: the LDOS sites, or the distinct from-indices
  // of a Green's-function request in order of first appearance
  std::vector<uint32_t> sites;
  // Green's-function pairs: to[k], and the source (index into sites) of pair k
  std::vector<uint32_t> to, pair_src;
  // some pair has to != from: every lane gathers all moments directly
  // (M - 1 steps) into pair slots instead of stepping to M/2 with doubling
  bool direct = false;
  std::vector<uint32_t> slots;  // pair slot of pair k in its model (direct requests)
  uint32_t M = 0;
  double broadening = 0;
  Clock::time_point t_submit;
  std::vector<uint32_t> lanes;
  int32_t base = 0;
  bool done = false;
  bool finishing = false;  // its results are being formed (cancel no longer applies)
  bool cancelled = false;
  int status = TBTKKPM_OK;
  std::string message;
  std::vector<double> ldos, err;  // LDOS [K][E], or G [K][E] complex for a GF request
  std::vector<int32_t> rerun;
  // staging of the finish phase
  size_t stage_off = 0;
  // recursion steps of each lane
  uint32_t steps() const { return direct ? M - 1 : M / 2; }
  // results: one per site, or one per pair
  uint32_t outputs() const { return kind == kLdos ? (uint32_t)sites.size() : (uint32_t)to.size(); }
  // doubles of one result over the energy grid
  uint32_t result_doubles(uint32_t E) const { return kind == kLdos ? E : 2 * E; }
};

struct Model {
  uint32_t id = 0;
  tbtkkpm_matrix *mat = nullptr;
  tbtkkpm_table *table = nullptr;  // the server's table of this scale
  // Wmax lanes are allocated; the steps run at width W, the smallest power
  // of two (at least kMinStepWidth) that covers every busy lane, or Wmax
  // when the width does not follow demand (tbtkkpm_server_set_adaptive_width)
  uint32_t N = 0, W = 0, Wmax = 0;
  double scale = 1;
  bool real = false;  // real Hamiltonian: lanes hold real float vectors
  uint32_t head_steps = 0;  // FP64 head of a lane (0: none)
  bool resident = false;
  uint64_t bytes = 0;
  uint64_t last_tick = 0;
  size_t esize() const { return real ? sizeof(float) : sizeof(float2); }
  DevBuf vec[2], dots, mu, mu_direct, base, laneM, bitmap, tlist, pmu;
  std::vector<int32_t> base_h;
  std::vector<uint32_t> M_h;
  std::vector<uint64_t> lane_req;  // request per lane, 0 when free
  std::vector<uint32_t> lane_site;
  // per lane: (to row, pair slot) of its Green's-function pairs (direct requests)
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> lane_pairs;
  std::vector<uint64_t> pair_req;  // request per pair slot, 0 when free
  std::vector<uint32_t> bitmap_h;
  uint32_t busy = 0, pairs_busy = 0;
  uint32_t tcount = 0;
  bool dirty = true;
  DevBuf lane_mem;  // one allocation; the lane buffers above are views into it
  // gather plans of the matrix by 2 * rows per tile + complex (null: none)
  std::map<int, const TilePlan *> plans;
  void release_lanes() {
    for (DevBuf *b : {&vec[0], &vec[1], &dots, &mu, &mu_direct, &base, &laneM, &bitmap, &tlist,
                      &pmu}) {
      b->ptr = nullptr;
      b->cap = 0;
    }
    lane_mem.release();
    resident = false;
  }
};

// The FP64 recomputation of the outputs `idx` of a finished request, with
// copies of what it needs: the rerun thread writes the results back under
// the server's lock, by request id, only if the request still waits.
struct RerunJob {
  uint64_t id = 0;
  Model *m = nullptr;
  int kind = kLdos;
  uint32_t M = 0;
  double broadening = 0;
  std::vector<uint32_t> sites, to, pair_src, idx;
};

// Lane memory of a model: vectors, fixed-point sums, moments, lane tables,
// target bitmap and list (a row and an entry word for each of up to W
// lane sites and W pair targets), pair moments.
uint64_t lane_bytes(uint32_t N, uint32_t W, uint32_t Mmax, uint32_t ld, size_t esize) {
  return 2ull * N * W * esize + 2ull * W * sizeof(long long) +
         (uint64_t)W * Mmax * sizeof(double2) + (uint64_t)W * ld * sizeof(double2) +
         8ull * W + 4ull * ((N + 31) / 32) + 16ull * W + (uint64_t)W * Mmax * sizeof(double2);
}

// The step kernels of one class (complex64 lanes or real float lanes):
// register-staged, then tile-staged entries.
const std::vector<const MultiEntry *> &multi_entries(bool real) {
  static const std::vector<const MultiEntry *> lists[2] = {
      [] {
        std::vector<const MultiEntry *> v;
        for (int i = 0; i < kNumMultiSteps; i++) v.push_back(&kMultiSteps[i]);
        for (int i = 0; i < kNumMultiTiled; i++) v.push_back(&kMultiTiled[i]);
        return v;
      }(),
      [] {
        std::vector<const MultiEntry *> v;
        for (int i = 0; i < kNumMultiStepsReal; i++) v.push_back(&kMultiStepsReal[i]);
        for (int i = 0; i < kNumMultiTiledReal; i++) v.push_back(&kMultiTiledReal[i]);
        return v;
      }()};
  return lists[real ? 1 : 0];
}

const MultiEntry *find_multi(int tpr, int vpt, int minb, bool real) {
  for (const MultiEntry *e : multi_entries(real))
    if (e->tpr == tpr && e->vpt == vpt && e->minb == minb) return e;
  return nullptr;
}

// Gather plan of a model for a tile-staged entry (built on first use on the
// model's matrix handle); null when the entry is register-staged, rows of W
// lanes are too narrow for bulk copies, or the matrix has a tile the plan
// builder cannot take.
const TilePlan *model_plan(Model *m, uint32_t W, const MultiEntry *e, int *rc) {
  *rc = TBTKKPM_OK;
  if (!is_multi_tiled(e->minb) || (W * m->esize()) % 16 != 0) return nullptr;
  const int R = multi_tiled_rows(e->minb), key = 2 * R + (m->real ? 0 : 1);
  auto it = m->plans.find(key);
  if (it != m->plans.end()) return it->second;
  // the first use builds it on the matrix handle (under its lock: the rerun
  // thread may be running an FP64 recomputation on the same handle)
  const TilePlan *p = nullptr;
  {
    std::lock_guard<std::mutex> lk(m->mat->lock);
    *rc = tile_plan(m->mat, R, !m->real, &p);
  }
  if (*rc) return nullptr;
  m->plans[key] = p;
  return p;
}

// Shared-memory ring of a tile-staged entry over models whose plans have
// at most wmax entries per row and umax outside rows per tile (stages 0:
// two stages do not fit).
TiledLayout multi_layout(const MultiEntry *e, uint32_t W, bool real, uint32_t wmax, uint32_t umax) {
  TilePlan p{};
  p.R = (uint32_t)multi_tiled_rows(e->minb);
  p.wmax = wmax;
  p.umax = umax;
  // the kernel's header holds a StageMeta per stage beside the barriers
  return tiled_layout(p, W * (uint32_t)(real ? sizeof(float) : sizeof(float2)),
                      real ? (uint32_t)sizeof(double) : (uint32_t)sizeof(double2),
                      tiled_budget(multi_tiled_bps(e->minb)) - (kMultiHeader - kTiledHeader));
}

// Default shape per width and class (measured choices of the single-model
// kernels: few threads per row, several values each).
std::array<int, 3> default_config(uint32_t W, bool real) {
  if (real) {
    switch (W) {
      case 1: return {1, 1, 2};
      case 2: return {1, 2, 2};
      case 4: return {1, 4, 2};
      case 8: return {1, 8, 2};
      case 16: return {4, 4, 2};
      case 32: return {8, 4, 2};
      default: return {8, 8, 2};
    }
  }
  switch (W) {
    case 1: return {1, 1, 2};
    case 2: return {2, 1, 2};
    case 4: return {2, 2, 2};
    case 8: return {4, 2, 2};
    case 16: return {8, 2, 2};
    case 32: return {8, 4, 2};
    default: return {8, 8, 2};
  }
}

}  // namespace
}  // namespace tbtkkpm

using namespace tbtkkpm;

struct tbtkkpm_server {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t Mmax = 0, E = 0, ld = 0;
  std::vector<double> energies;
  uint64_t budget = 0;
  uint32_t tick_steps = 64;
  double tol = 0;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::unique_ptr<Model>> models;
  std::map<double, tbtkkpm_table *> tables;                         // Mmax rows per scale
  std::map<uint32_t, std::array<int, 3>> config;  // width | real << 16 -> tpr, vpt, minb
  std::set<uint32_t> tuned;                       // keys of config the autotuner measured
  bool use_real = true;                           // real lanes for real models added later
  uint32_t head_steps = kPrefixSteps;             // FP64 head of models added later
  bool table_free = false;                        // Clenshaw energy sums for scales added later
  uint32_t wait_limit = kWaitLimit;               // polls per staged-row wait (set_wait_limit)
  bool adaptive_width = true;                     // step widths follow demand (set_adaptive_width)
  Workspace head_ws;                              // FP64 head scratch (worker thread)
  std::deque<uint64_t> pending;
  std::map<uint64_t, std::unique_ptr<Request>> requests;
  uint64_t next_id = 1;
  bool stop = false;
  bool working = false;  // a tick or finish phase is running
  // FP64 recomputations run on their own thread (rerun_worker), so the
  // worker keeps stepping the other requests meanwhile
  // (kRerunThreads threads: the FP64 recomputations of small models are
  // launch-bound, so several run side by side on their own streams)
  static constexpr int kRerunThreads = 4;
  std::deque<RerunJob> rerun_jobs;
  int rerun_running = 0;
  std::condition_variable cv_rerun;
  std::thread rerun_threads[kRerunThreads];
  int failed = 0;
  std::string fail_msg;
  std::thread worker;

  int32_t n_global = 1;  // next global step
  uint64_t tick_no = 0;
  uint64_t resident = 0;
  DevBuf d_models, d_hdr, d_joins, d_done, d_pairs, d_stage, d_damp, d_tiles, d_tdesc, d_truns;
  DevBuf d_err;           // staged-row wait that ran out (tile-staged steps)
  int *h_err = nullptr;   // pinned copy of d_err read after each tick
  // statistics
  std::vector<double> latencies_ms;
  double reruns = 0, ticks = 0, steps = 0, lane_steps = 0, evictions = 0, waited = 0, busy_s = 0;
  double step_s = 0, step_bytes = 0, finish_s = 0, rerun_s = 0, join_s = 0, plan_s = 0, tick_s = 0;
  double graph_ticks = 0, relayouts = 0;
  DevBuf d_res;                 // finish results of a tick: [ldos K*E | err K] per request
  double *h_res = nullptr;      // pinned host copy of d_res
  size_t h_res_cap = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};  // around the steps of a tick
  // The lane classes of a tick are independent (different models), so
  // their steps run on their own streams, forked from and joined back into
  // `stream`: a class of small, latency-bound steps overlaps the others.
  static constexpr int kClassStreams = 4;
  cudaStream_t cls_stream[kClassStreams] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kClassStreams] = {};
  // Each tick's steps replay a captured CUDA graph of one step of every
  // class (tick_exec; d_step counts the replays); off when a capture failed.
  bool use_graphs = true;
  cudaGraphExec_t tick_exec = nullptr;
  DevBuf d_step;

  const std::array<int, 3> &config_for(uint32_t W, bool real) {
    const uint32_t key = W | (real ? 1u << 16 : 0u);
    auto it = config.find(key);
    if (it == config.end()) it = config.emplace(key, default_config(W, real)).first;
    return it->second;
  }
};

namespace tbtkkpm {
namespace {

// ------------------------------------------------------------ admission

int make_resident(tbtkkpm_server *s, Model *m) {
  const uint32_t W = m->Wmax, N = m->N;
  const size_t words = (N + 31) / 32;
  int rc;
  const size_t es = m->esize();
  // one allocation per model for the ten lane buffers
  constexpr int kViews = 10;
  DevBuf *views[kViews] = {&m->vec[0], &m->vec[1], &m->dots,   &m->mu,    &m->mu_direct,
                           &m->base,   &m->laneM,  &m->bitmap, &m->tlist, &m->pmu};
  const size_t sizes[kViews] = {es * (size_t)N * W,
                                es * (size_t)N * W,
                                2 * sizeof(long long) * W,
                                sizeof(double2) * (size_t)W * s->Mmax,
                                sizeof(double2) * (size_t)W * s->ld,
                                4 * (size_t)W,
                                4 * (size_t)W,
                                4 * words,
                                16 * (size_t)W,
                                sizeof(double2) * (size_t)W * s->Mmax};
  size_t off[kViews], total = 0;
  for (int i = 0; i < kViews; i++) {
    off[i] = total;
    total += (sizes[i] + 255) & ~(size_t)255;
  }
  if ((rc = m->lane_mem.reserve(total))) {
    m->release_lanes();
    return rc;
  }
  for (int i = 0; i < kViews; i++) {
    views[i]->ptr = m->lane_mem.as<char>() + off[i];
    views[i]->cap = sizes[i];
  }
  cudaError_t e;
  if ((e = cudaMemsetAsync(m->vec[0].ptr, 0, es * (size_t)N * W, s->stream)) ||
      (e = cudaMemsetAsync(m->vec[1].ptr, 0, es * (size_t)N * W, s->stream)) ||
      (e = cudaMemsetAsync(m->dots.ptr, 0, 2 * sizeof(long long) * W, s->stream))) {
    m->release_lanes();
    return cuda_fail(e, "server: lane memory");
  }
  m->base_h.assign(W, kLaneIdle);
  m->M_h.assign(W, 0);
  m->lane_req.assign(W, 0);
  m->lane_site.assign(W, 0);
  m->lane_pairs.assign(W, {});
  m->pair_req.assign(W, 0);
  m->bitmap_h.assign(words, 0);
  m->busy = 0;
  m->pairs_busy = 0;
  m->W = m->Wmax;
  m->dirty = true;
  m->resident = true;
  s->resident += m->bytes;
  return TBTKKPM_OK;
}

void evict(tbtkkpm_server *s, Model *m) {
  cudaStreamSynchronize(s->stream);
  m->release_lanes();
  s->resident -= m->bytes;
  s->evictions += 1;
}

// Room for `need` more bytes: idle resident models leave, least recently
// used first.  False if the busy ones alone leave no room.
bool make_room(tbtkkpm_server *s, uint64_t need, const Model *keep) {
  while (s->resident + need > s->budget) {
    Model *victim = nullptr;
    for (auto &p : s->models) {
      Model *m = p.get();
      if (m == keep || !m->resident || m->busy) continue;
      if (!victim || m->last_tick < victim->last_tick) victim = m;
    }
    if (!victim) return false;
    evict(s, victim);
  }
  return true;
}

// A lane joining at this step boundary.
struct JoinRef {
  Model *m;
  uint32_t c;
  Request *r;
};

// A change of a model's step width at a step boundary: its two lane
// buffers are restrided in place (run_relayouts) before the joins run.
struct Relayout {
  Model *m;
  uint32_t from, to;
};

// The width model m steps at: the smallest power of two, at least
// kMinStepWidth, that covers its highest busy lane (Wmax when the width does
// not follow demand).
uint32_t step_width(const tbtkkpm_server *s, const Model *m) {
  if (!s->adaptive_width) return m->Wmax;
  uint32_t hi = 0;
  for (uint32_t c = 0; c < m->Wmax; c++)
    if (m->lane_req[c]) hi = c + 1;
  uint32_t w = std::min(kMinStepWidth, m->Wmax);
  while (w < hi) w *= 2;
  return w;
}

// Under s->mu.  Queued requests take free lanes in arrival order (the
// lowest free lanes of their model); the joins of this step boundary are
// appended (the lane bases assume no FP64 head until run_joins has reported
// the heads).  Then every resident model takes its step width: `moves` gets
// the restrides of models whose lanes already held state.
int admit(tbtkkpm_server *s, std::vector<MultiJoin> &joins, std::vector<JoinRef> &refs,
          std::vector<Relayout> &moves) {
  std::vector<uint32_t> busy0(s->models.size());
  for (size_t i = 0; i < s->models.size(); i++) busy0[i] = s->models[i]->busy;
  for (auto it = s->pending.begin(); it != s->pending.end();) {
    Request *r = s->requests.at(*it).get();
    Model *m = s->models[r->model].get();
    const uint32_t K = (uint32_t)r->sites.size();
    const uint32_t npairs = r->direct ? (uint32_t)r->to.size() : 0u;
    if (m->resident && (m->Wmax - m->busy < K || m->Wmax - m->pairs_busy < npairs)) {
      ++it;
      continue;
    }
    if (!m->resident) {
      if (!make_room(s, m->bytes, m)) {
        s->waited += 1;
        ++it;
        continue;
      }
      int rc = make_resident(s, m);
      if (rc == TBTKKPM_ERR_MEMORY) {
        s->waited += 1;
        ++it;
        continue;
      }
      if (rc) return rc;
    }
    r->base = s->n_global - 1;
    for (uint32_t c = 0, k = 0; c < m->Wmax && k < K; c++) {
      if (m->lane_req[c]) continue;
      const uint32_t site = r->sites[k++];
      m->lane_req[c] = r->id;
      m->lane_site[c] = site;
      m->base_h[c] = r->base;
      m->M_h[c] = r->M | (r->direct ? kDirectLane : 0u);
      m->bitmap_h[site >> 5] |= 1u << (site & 31);
      r->lanes.push_back(c);
      MultiJoin j;
      j.x = m->vec[(s->n_global + 1) & 1].as<float2>();
      j.mu = m->mu.as<double2>() + (size_t)c * s->Mmax;
      j.mu_direct = m->mu_direct.as<double2>() + (size_t)c * s->ld;
      j.rows = m->N;
      j.col = c;
      j.site = site;
      j.W = m->W;
      j.real = m->real ? 1u : 0u;
      j.x_prev = m->vec[s->n_global & 1].as<float2>();
      j.M = r->M;
      joins.push_back(j);
      refs.push_back({m, c, r});
    }
    if (r->direct) {
      // pair slots: pair k's moments are gathered at its to-row from its
      // source's lane
      r->slots.clear();
      for (uint32_t k = 0, d = 0; k < npairs; k++) {
        while (m->pair_req[d]) d++;
        m->pair_req[d] = r->id;
        m->lane_pairs[r->lanes[r->pair_src[k]]].push_back({r->to[k], d});
        r->slots.push_back(d);
      }
      m->pairs_busy += npairs;
    }
    m->busy += K;
    m->dirty = true;
    it = s->pending.erase(it);
  }
  for (size_t i = 0; i < s->models.size(); i++) {
    Model *m = s->models[i].get();
    if (!m->resident || !m->busy) continue;
    const uint32_t w = step_width(s, m);
    if (w == m->W) continue;
    if (busy0[i]) moves.push_back({m, m->W, w});
    m->W = w;
    m->dirty = true;
  }
  for (size_t i = 0; i < joins.size(); i++) joins[i].W = refs[i].m->W;
  return TBTKKPM_OK;
}

// Restrides the lane buffers of `moves` on the server's stream (worker
// thread, no lock held; the previous tick has ended, the joins follow).
int run_relayouts(tbtkkpm_server *s, const std::vector<Relayout> &moves) {
  std::vector<std::pair<uint32_t, uint32_t>> ranges;
  uint64_t launches = 0;
  for (const Relayout &mv : moves) {
    const Model *m = mv.m;
    lane_relayout_ranges(m->N, mv.from, mv.to, ranges);
    for (int b = 0; b < 2; b++)
      for (const auto &rg : ranges) {
        const uint64_t n = (uint64_t)(rg.second - rg.first) * mv.to;
        const unsigned grid = (unsigned)std::min<uint64_t>(blocks_for(n), 8ull * sm_count(s->device));
        if (m->real)
          kpm_lane_relayout<float><<<grid, 256, 0, s->stream>>>(m->vec[b].as<float>(), rg.first,
                                                                rg.second, mv.from, mv.to);
        else
          kpm_lane_relayout<float2><<<grid, 256, 0, s->stream>>>(m->vec[b].as<float2>(), rg.first,
                                                                 rg.second, mv.from, mv.to);
        launches += 1;
      }
  }
  count_launches(launches);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "server: lane restride");
  return TBTKKPM_OK;
}

// Frees the lanes and pair slots of a request that finished or was
// cancelled (under s->mu).
void release_request_lanes(Model *m, Request *r) {
  for (uint32_t c : r->lanes) {
    m->lane_req[c] = 0;
    m->base_h[c] = kLaneIdle;
    m->M_h[c] = 0;
    m->lane_pairs[c].clear();
  }
  for (uint32_t d : r->slots) m->pair_req[d] = 0;
  m->pairs_busy -= (uint32_t)r->slots.size();
  m->busy -= (uint32_t)r->lanes.size();
  m->dirty = true;
}

// ------------------------------------------------------------ one tick

struct ClassPlan {
  uint32_t W;
  bool real = false;
  const MultiEntry *entry;
  std::vector<MultiModel> models;
  uint32_t total_tiles = 0;
  uint32_t total_runs = 0;  // tile-staged entries: runs of the launch
  TiledLayout ly{};         // tile-staged entries: the class's ring
  double bytes = 0;         // algorithmic bytes of one step
};

// Uploads the lane tables and targets of changed models (under s->mu; the
// copies come from pageable memory, so the host arrays are free on return).
int upload_lanes(tbtkkpm_server *s, Model *m) {
  if (!m->dirty) return TBTKKPM_OK;
  // target list sorted by row: every busy lane at its site (direct
  // moments of its own source), and the pair targets of direct lanes
  std::vector<std::pair<uint32_t, uint32_t>> t;
  std::fill(m->bitmap_h.begin(), m->bitmap_h.end(), 0u);
  for (uint32_t c = 0; c < m->Wmax; c++)
    if (m->lane_req[c]) {
      t.push_back({m->lane_site[c], c});
      for (const auto &pr : m->lane_pairs[c]) t.push_back({pr.first, c | (pr.second << 8) | kPairEntry});
    }
  for (const auto &e : t) m->bitmap_h[e.first >> 5] |= 1u << (e.first & 31);
  std::sort(t.begin(), t.end());
  const size_t cap = 2 * (size_t)m->Wmax;
  std::vector<uint32_t> tl(2 * cap, 0);
  for (size_t i = 0; i < t.size(); i++) {
    tl[i] = t[i].first;
    tl[cap + i] = t[i].second;
  }
  m->tcount = (uint32_t)t.size();
  // the four tables are adjacent views of the lane memory: one copy of the
  // range from base to the end of tlist (alignment gaps included)
  char *lo = m->base.as<char>();
  const size_t range = (size_t)(m->tlist.as<char>() - lo) + 4 * tl.size();
  std::vector<char> buf(range, 0);
  auto put = [&](const DevBuf &v, const void *src, size_t n) {
    std::memcpy(buf.data() + (v.as<char>() - lo), src, n);
  };
  put(m->base, m->base_h.data(), 4 * (size_t)m->Wmax);
  put(m->laneM, m->M_h.data(), 4 * (size_t)m->Wmax);
  put(m->bitmap, m->bitmap_h.data(), 4 * m->bitmap_h.size());
  put(m->tlist, tl.data(), 4 * tl.size());
  cudaError_t e;
  if ((e = cudaMemcpyAsync(lo, buf.data(), range, cudaMemcpyHostToDevice, s->stream)))
    return cuda_fail(e, "server: lane tables");
  m->dirty = false;
  return TBTKKPM_OK;
}

MultiModel describe(const tbtkkpm_server *s, const Model *m) {
  MultiModel d{};
  d.A.slice_ptr = m->mat->slice_ptr.as<uint32_t>();
  d.A.col = m->mat->scol.as<uint32_t>();
  d.A.val = m->mat->sval.as<double2>();
  d.A.vre = m->real ? m->mat->sreal.as<double>() : nullptr;
  d.A.N = m->N;
  d.A.nslices = m->mat->nslices;
  d.vec[0] = m->vec[0].as<float2>();
  d.vec[1] = m->vec[1].as<float2>();
  d.bitmap = m->bitmap.as<uint32_t>();
  d.trow = m->tlist.as<uint32_t>();
  d.tcol = m->tlist.as<uint32_t>() + 2 * m->Wmax;
  d.tcount = m->tcount;
  d.base = m->base.as<int32_t>();
  d.lane_M = m->laneM.as<uint32_t>();
  d.dots = m->dots.as<long long>();
  d.mu = m->mu.as<double2>();
  d.mu_direct = m->mu_direct.as<double2>();
  d.pmu = m->pmu.as<double2>();
  d.mmax = s->Mmax;
  return d;
}

// Builds the launch plans, one per (lane width, real or complex lanes), of
// all models with busy lanes (under s->mu).  A class whose configured entry
// is tile-staged falls back to the default register-staged entry of its
// width when some model has no plan for it or two ring stages do not fit.
int plan_tick(tbtkkpm_server *s, std::vector<ClassPlan> &plans) {
  std::map<uint32_t, size_t> index;
  std::vector<std::vector<Model *>> members;
  for (auto &p : s->models) {
    Model *m = p.get();
    if (!m->resident || !m->busy) continue;
    int rc = upload_lanes(s, m);
    if (rc) return rc;
    m->last_tick = s->tick_no;
    const uint32_t key = m->W | (m->real ? 1u << 16 : 0u);
    auto it = index.find(key);
    if (it == index.end()) {
      const auto &cfg = s->config_for(m->W, m->real);
      ClassPlan cp;
      cp.W = m->W;
      cp.real = m->real;
      cp.entry = find_multi(cfg[0], cfg[1], cfg[2], m->real);
      if (!cp.entry)
        return fail(TBTKKPM_ERR_UNSUPPORTED, "server: no step kernel for width %u", m->W);
      it = index.emplace(key, plans.size()).first;
      plans.push_back(std::move(cp));
      members.emplace_back();
    }
    members[it->second].push_back(m);
  }
  for (size_t c = 0; c < plans.size(); c++) {
    ClassPlan &cp = plans[c];
    std::vector<const TilePlan *> tp(members[c].size(), nullptr);
    if (is_multi_tiled(cp.entry->minb)) {
      uint32_t wmax = 0, umax = 0;
      bool ok = true;
      for (size_t i = 0; i < members[c].size() && ok; i++) {
        int rc;
        tp[i] = model_plan(members[c][i], cp.W, cp.entry, &rc);
        if (rc) return rc;
        ok = tp[i] != nullptr;
        if (ok) {
          wmax = std::max(wmax, tp[i]->wmax);
          umax = std::max(umax, tp[i]->umax);
        }
      }
      if (ok) cp.ly = multi_layout(cp.entry, cp.W, cp.real, wmax, umax);
      if (!ok || cp.ly.stages == 0) {
        const auto d = default_config(cp.W, cp.real);
        cp.entry = find_multi(d[0], d[1], d[2], cp.real);
        std::fill(tp.begin(), tp.end(), nullptr);
      }
    }
    for (size_t i = 0; i < members[c].size(); i++) {
      const Model *m = members[c][i];
      MultiModel d = describe(s, m);
      d.tile0 = cp.total_tiles;
      if (tp[i]) {
        d.ntiles = tp[i]->ntiles;
        d.p_hdr = tp[i]->hdr;
        d.p_runs = tp[i]->runs;
        d.p_slot = tp[i]->eslot;
        d.p_val = tp[i]->eval;
        d.p_nruns = tp[i]->nruns;
        d.run0 = cp.total_runs;
        cp.total_runs += tp[i]->nruns;
      } else {
        const uint32_t rpb = kBlock / cp.entry->tpr;
        d.ntiles = (uint32_t)(((uint64_t)m->mat->nslices * 32 + rpb - 1) / rpb);
      }
      cp.total_tiles += d.ntiles;
      // matrix once (value + column index, row pointers) and three vector
      // passes of the lanes
      cp.bytes += (m->real ? 12.0 : 20.0) * m->mat->nnz + 4.0 * (m->N + 1) +
                  3.0 * m->N * m->W * m->esize();
      cp.models.push_back(d);
    }
  }
  return TBTKKPM_OK;
}

// Starts the lanes of `joins` at global step s->n_global (worker thread, no
// lock held): clears their columns and moment rows, then runs the FP64 head
// of every lane whose model has one, which writes j_q, j_{q-1} into its
// columns; head[i] = q of join i (0: plain start from j_0).  Returns after
// the stream has passed the joins.
int run_joins(tbtkkpm_server *s, const std::vector<MultiJoin> &joins, const std::vector<JoinRef> &refs,
              std::vector<uint32_t> &head) {
  cudaStream_t st = s->stream;
  int rc;
  cudaError_t e;
  head.assign(joins.size(), 0);
  if (joins.empty()) return TBTKKPM_OK;
  if ((rc = s->d_joins.reserve(sizeof(MultiJoin) * joins.size()))) return rc;
  if ((e = cudaMemcpyAsync(s->d_joins.ptr, joins.data(), sizeof(MultiJoin) * joins.size(),
                           cudaMemcpyHostToDevice, st)))
    return cuda_fail(e, "server: joins");
  uint32_t rows = 0;
  for (const MultiJoin &j : joins) rows = std::max(rows, j.rows);
  const unsigned bx = std::max(1u, std::min(blocks_for(std::max(rows, s->Mmax)), 512u));
  for (size_t j0 = 0; j0 < joins.size(); j0 += 65535) {
    const unsigned nj = (unsigned)std::min<size_t>(65535, joins.size() - j0);
    kpm_multi_join<<<dim3(bx, nj), 256, 0, st>>>(s->d_joins.as<MultiJoin>() + j0, s->Mmax, s->ld);
  }
  count_launches((joins.size() + 65534) / 65535);
  std::vector<PrefixJob> jobs;
  std::vector<size_t> which;
  for (size_t i = 0; i < joins.size(); i++) {
    const MultiJoin &j = joins[i];
    const Model *m = refs[i].m;
    const uint32_t want = std::min(m->head_steps, j.M / 2 >= 1 ? j.M / 2 - 1 : 0u);
    // the head writes its source's own moments only: lanes that gather
    // pair moments start from j_0
    if (!m->mat->pattern_symmetric || want < 2 || refs[i].r->direct) continue;
    PrefixJob p{};
    p.slice_ptr = m->mat->slice_ptr.as<uint32_t>();
    p.scol = m->mat->scol.as<uint32_t>();
    p.sval = m->mat->sval.as<double2>();
    p.site = j.site;
    p.steps = want;
    p.M = j.M;
    p.ld = s->ld;
    p.mu = j.mu;
    p.mu_direct = j.mu_direct;
    p.x_cur = j.x;
    p.x_prev = j.x_prev;
    p.W = j.W;
    p.col = j.col;
    p.real = j.real;
    jobs.push_back(p);
    which.push_back(i);
  }
  std::vector<PrefixResult> res;
  if ((rc = run_fp64_head(st, jobs, s->head_ws, res))) return rc;
  for (size_t k = 0; k < which.size(); k++) head[which[k]] = res[k].q >= 2 ? res[k].q : 0;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "server: joins");
  return TBTKKPM_OK;
}

// Launches `nsteps` steps of every plan starting at global step s->n_global
// (worker thread, no lock held).
int run_tick(tbtkkpm_server *s, const std::vector<ClassPlan> &plans, uint32_t nsteps) {
  cudaStream_t st = s->stream;
  int rc;
  cudaError_t e;
  // descriptors and headers of all plans in one upload
  size_t nm = 0;
  for (const ClassPlan &cp : plans) nm += cp.models.size();
  std::vector<MultiModel> all;
  all.reserve(nm);
  std::vector<MultiHeader> hdr;
  size_t tiles = 0, runs = 0;
  for (const ClassPlan &cp : plans) {
    tiles += cp.total_tiles;
    runs += cp.total_runs;
  }
  if ((rc = s->d_tiles.reserve(sizeof(uint32_t) * std::max<size_t>(tiles, 1))) ||
      (rc = s->d_tdesc.reserve(sizeof(uint4) * kDescWords * std::max<size_t>(tiles, 1))) ||
      (rc = s->d_truns.reserve(sizeof(uint2) * std::max<size_t>(runs, 1))))
    return rc;
  tiles = runs = 0;
  for (const ClassPlan &cp : plans) {
    all.insert(all.end(), cp.models.begin(), cp.models.end());
    // tile-staged launches: runs of 8-32 tiles per block, long enough that
    // a block rarely changes model, short enough that every block has work
    uint32_t run = kRun;
    if (is_multi_tiled(cp.entry->minb)) {
      const uint32_t grid = (uint32_t)multi_tiled_bps(cp.entry->minb) * (uint32_t)sm_count(s->device);
      run = std::max(kRun, std::min(32u, cp.total_tiles / std::max(4 * grid, 1u)));
    }
    hdr.push_back({(uint32_t)cp.models.size(), cp.total_tiles, s->n_global,
                   s->d_tiles.as<uint32_t>() + tiles, s->d_tdesc.as<uint4>() + kDescWords * tiles,
                   s->d_truns.as<uint2>() + runs, run, s->use_graphs ? s->d_step.as<int32_t>() : nullptr});
    tiles += cp.total_tiles;
    runs += cp.total_runs;
  }
  if ((rc = s->d_models.reserve(sizeof(MultiModel) * std::max<size_t>(nm, 1))) ||
      (rc = s->d_hdr.reserve(sizeof(MultiHeader) * std::max<size_t>(hdr.size(), 1))))
    return rc;
  if ((e = cudaMemcpyAsync(s->d_models.ptr, all.data(), sizeof(MultiModel) * nm,
                           cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(s->d_hdr.ptr, hdr.data(), sizeof(MultiHeader) * hdr.size(),
                           cudaMemcpyHostToDevice, st)))
    return cuda_fail(e, "server: descriptors");
  {
    size_t off = 0;
    for (size_t p = 0; p < plans.size(); p++) {
      const MultiModel *dm = s->d_models.as<MultiModel>() + off;
      const MultiHeader &h = hdr[p];
      if (is_multi_tiled(plans[p].entry->minb))
        kpm_multi_tilemap_tiled<<<(unsigned)plans[p].models.size(), 256, 0, st>>>(
            dm, s->d_hdr.as<MultiHeader>() + p, (uint32_t)multi_tiled_rows(plans[p].entry->minb),
            const_cast<uint4 *>(h.tile_desc), const_cast<uint2 *>(h.tile_runs));
      else
        kpm_multi_tilemap<<<(unsigned)plans[p].models.size(), 256, 0, st>>>(
            dm, s->d_hdr.as<MultiHeader>() + p, const_cast<uint32_t *>(h.tile_model));
      off += plans[p].models.size();
    }
    count_launches(plans.size());
  }
  // class p steps on stream p % kClassStreams (in order within a class):
  // the launches of `steps` steps from step offset k0, forked from st and
  // joined back into it
  const int nstreams = (int)std::min<size_t>(plans.size(), tbtkkpm_server::kClassStreams);
  auto launch_steps = [&](uint32_t k0, uint32_t steps) -> cudaError_t {
    cudaError_t ee;
    if (nstreams > 1) {
      if ((ee = cudaEventRecord(s->ev_fork, st))) return ee;
      for (int i = 0; i < nstreams; i++)
        if ((ee = cudaStreamWaitEvent(s->cls_stream[i], s->ev_fork, 0))) return ee;
    }
    for (uint32_t k = k0; k < k0 + steps; k++) {
      size_t off = 0;
      for (size_t p = 0; p < plans.size(); p++) {
        const ClassPlan &cp = plans[p];
        const MultiModel *dm = s->d_models.as<MultiModel>() + off;
        const MultiHeader *dh = s->d_hdr.as<MultiHeader>() + p;
        cudaStream_t cs = nstreams > 1 ? s->cls_stream[p % nstreams] : st;
        cp.entry->launch(cs, s->device, dm, dh, k, cp.W, s->ld,
                         MultiLaunch{cp.ly, s->d_err.as<int>(), s->wait_limit});
        kpm_multi_finalize<<<(unsigned)cp.models.size(), std::min<uint32_t>(std::max(cp.W, 32u), 64u),
                             0, cs>>>(dm, dh, k, cp.W, s->Mmax, s->ld);
        off += cp.models.size();
      }
    }
    if (nstreams > 1)
      for (int i = 0; i < nstreams; i++)
        if ((ee = cudaEventRecord(s->ev_join[i], s->cls_stream[i])) ||
            (ee = cudaStreamWaitEvent(st, s->ev_join[i], 0)))
          return ee;
    return cudaGetLastError();
  };
  // The tick's graph: one step of every class, captured once and replayed
  // nsteps times (the device counter d_step gives each replay its step).
  // A capture or instantiation that fails falls back to direct launches.
  if (s->tick_exec) {
    cudaGraphExecDestroy(s->tick_exec);
    s->tick_exec = nullptr;
  }
  // the headers of this tick read d_step when graphs are on: it starts at 0
  if (hdr[0].step && (e = cudaMemsetAsync(s->d_step.ptr, 0, sizeof(int32_t), st)))
    return cuda_fail(e, "server: step counter");
  bool replay = false;
  if (hdr[0].step && nsteps > 1) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
      cudaError_t ce = launch_steps(0, 1);
      if (ce == cudaSuccess) {
        kpm_multi_advance<<<1, 32, 0, st>>>(s->d_step.as<int32_t>());
        ce = cudaGetLastError();
      }
      const cudaError_t ee = cudaStreamEndCapture(st, &g);
      if (ce == cudaSuccess && ee == cudaSuccess && g &&
          cudaGraphInstantiate(&s->tick_exec, g, 0) == cudaSuccess)
        replay = true;
      if (g) cudaGraphDestroy(g);
    }
    cudaGetLastError();
    if (!replay) s->use_graphs = false;  // direct launches from the next tick on
  }
  cudaEventRecord(s->ev[0], st);
  if (replay) {
    for (uint32_t k = 0; k < nsteps; k++)
      if ((e = cudaGraphLaunch(s->tick_exec, st))) return cuda_fail(e, "server: step graph");
  } else if ((e = launch_steps(0, nsteps))) {
    return cuda_fail(e, "server: step launch");
  }
  cudaEventRecord(s->ev[1], st);
  count_launches((2ull * plans.size() + (replay ? 1 : 0)) * nsteps);
  if (replay) s->graph_ticks += 1;
  if ((e = cudaGetLastError())) return cuda_fail(e, "server: step launch");
  // the wait flag of the tile-staged steps, read after the tick
  if ((e = cudaMemcpyAsync(s->h_err, s->d_err.ptr, sizeof(int), cudaMemcpyDeviceToHost, st)))
    return cuda_fail(e, "server: step status");
  return TBTKKPM_OK;
}

// ------------------------------------------------------------ finish

// The finish phase of the requests that completed in one tick, in two
// halves: finish_launch enqueues their damping, energy sums and error
// estimates and the copy of all results into pinned memory on the server's
// stream (before any later join can reuse their lanes); finish_complete
// waits for that copy, fills the requests and runs the FP64 recomputations
// of the sites past the tolerance.  The worker runs the second half while
// the next tick's steps are on the device.
struct FinishBatch {
  std::vector<Request *> done;
  std::vector<Model *> owner;
  std::vector<size_t> res_off;  // offset of each request's results in h_res
  cudaEvent_t ev = nullptr;     // after the results copy
  // FP64 recomputations the host half found, and their requests (which
  // complete when the rerun thread has written them back)
  std::vector<RerunJob> reruns;
  std::vector<Request *> rerun_req;
};

int finish_launch(tbtkkpm_server *s, FinishBatch &fb) {
  if (fb.done.empty()) return TBTKKPM_OK;
  cudaStream_t st = s->stream;
  const uint32_t E = s->E;
  // moments stage per request: damped moments [K][M] of its K outputs;
  // results per request: LDOS [K][E] or G [K][E] complex, then err [K]
  size_t total = 0, lanes = 0, pairs = 0, damp_len = 0, nres = 0;
  fb.res_off.resize(fb.done.size());
  for (size_t i = 0; i < fb.done.size(); i++) {
    Request *r = fb.done[i];
    const size_t K = r->outputs(), M = r->M;
    r->stage_off = total;
    total += sizeof(double2) * K * M;
    total = (total + 255) & ~(size_t)255;
    nres = (nres + 1) & ~(size_t)1;  // complex results start on 16 bytes
    fb.res_off[i] = nres;
    nres += K * r->result_doubles(E) + K;
    (r->direct ? pairs : lanes) += K;
    damp_len += M;
  }
  int rc;
  if ((rc = s->d_stage.reserve(total)) ||
      (rc = s->d_done.reserve(sizeof(MultiDone) * std::max<size_t>(lanes, 1))) ||
      (rc = s->d_pairs.reserve(sizeof(MultiPair) * std::max<size_t>(pairs, 1))) ||
      (rc = s->d_damp.reserve(sizeof(double) * damp_len)) || (rc = s->d_res.reserve(sizeof(double) * nres)))
    return rc;
  cudaError_t e;
  if (s->h_res_cap < nres) {
    if (s->h_res) cudaFreeHost(s->h_res);
    s->h_res = nullptr;
    s->h_res_cap = 0;
    const size_t cap = std::max(nres + nres / 2, (size_t)1 << 20);
    if ((e = cudaMallocHost(&s->h_res, sizeof(double) * cap)) != cudaSuccess)
      return cuda_fail(e, "server: pinned results");
    s->h_res_cap = cap;
  }
  // per output: the moment rows of its lane (LDOS sites, diagonal pairs)
  // or its pair slot (direct requests)
  std::vector<MultiDone> lane_ptr;
  std::vector<MultiPair> pair_ptr;
  std::vector<double> damp_all;
  std::vector<double> bvals;
  for (size_t i = 0; i < fb.done.size(); i++) {
    Request *r = fb.done[i];
    Model *m = fb.owner[i];
    auto lane_rows = [&](uint32_t c) {
      return MultiDone{m->mu.as<double2>() + (size_t)c * s->Mmax,
                       m->mu_direct.as<double2>() + (size_t)c * s->ld};
    };
    if (r->kind == kLdos) {
      for (uint32_t c : r->lanes) lane_ptr.push_back(lane_rows(c));
    } else if (!r->direct) {
      for (uint32_t k = 0; k < r->to.size(); k++) lane_ptr.push_back(lane_rows(r->lanes[r->pair_src[k]]));
    } else {
      for (uint32_t k = 0; k < r->to.size(); k++) {
        const MultiDone l = lane_rows(r->lanes[r->pair_src[k]]);
        pair_ptr.push_back({m->pmu.as<double2>() + (size_t)r->slots[k] * s->Mmax,
                            r->to[k] == r->sites[r->pair_src[k]] ? 1.0 : 0.0, l.mu, l.mu_direct});
      }
    }
    std::vector<double> a;
    double b = 1;
    if (r->broadening != 0) damping_factors(r->M, r->broadening, a, b);
    else a.assign(r->M, 1.0);
    damp_all.insert(damp_all.end(), a.begin(), a.end());
    bvals.push_back(b);
  }
  if ((!lane_ptr.empty() &&
       (e = cudaMemcpyAsync(s->d_done.ptr, lane_ptr.data(), sizeof(MultiDone) * lane_ptr.size(),
                            cudaMemcpyHostToDevice, st))) ||
      (!pair_ptr.empty() &&
       (e = cudaMemcpyAsync(s->d_pairs.ptr, pair_ptr.data(), sizeof(MultiPair) * pair_ptr.size(),
                            cudaMemcpyHostToDevice, st))) ||
      (e = cudaMemcpyAsync(s->d_damp.ptr, damp_all.data(), sizeof(double) * damp_len,
                           cudaMemcpyHostToDevice, st)))
    return cuda_fail(e, "server: finish staging");
  size_t lane0 = 0, pair0 = 0, d0 = 0;
  for (size_t i = 0; i < fb.done.size(); i++) {
    Request *r = fb.done[i];
    Model *m = fb.owner[i];
    const uint32_t K = r->outputs(), M = r->M;
    double2 *out = reinterpret_cast<double2 *>(s->d_stage.as<char>() + r->stage_off);
    double *res = s->d_res.as<double>() + fb.res_off[i];
    double *err = res + (size_t)K * r->result_doubles(E);
    if (r->direct) {
      const MultiPair *pp = s->d_pairs.as<MultiPair>() + pair0;
      kpm_multi_prepare_pairs<<<blocks_for((uint64_t)K * M), 256, 0, st>>>(
          pp, K, M, s->d_damp.as<double>() + d0, bvals[i], r->broadening != 0, out);
      kpm_pair_error<<<K, kErrorBlock, 0, st>>>(pp, M, err);
      pair0 += K;
    } else {
      const MultiDone *dd = s->d_done.as<MultiDone>() + lane0;
      kpm_multi_prepare<<<blocks_for((uint64_t)K * M), 256, 0, st>>>(
          dd, K, M, s->d_damp.as<double>() + d0, bvals[i], r->broadening != 0, out, nullptr, nullptr);
      kpm_multi_error<<<K, kErrorBlock, 0, st>>>(dd, M, err);
      lane0 += K;
    }
    count_launches(2);
    // LDOS (4) or the request's Green's function type
    if ((rc = launch_energy_sum(st, m->table, out, K, r->kind == kLdos ? 4 : r->kind, res, M))) return rc;
    d0 += M;
  }
  if (!fb.ev && (e = cudaEventCreateWithFlags(&fb.ev, cudaEventDisableTiming)) != cudaSuccess)
    return cuda_fail(e, "server: finish event");
  if ((e = cudaMemcpyAsync(s->h_res, s->d_res.ptr, sizeof(double) * nres, cudaMemcpyDeviceToHost, st)) ||
      (e = cudaEventRecord(fb.ev, st)))
    return cuda_fail(e, "server: finish");
  return TBTKKPM_OK;
}

// FP64 recomputation of a job's outputs (rerun thread, no lock held): LDOS
// sites through the LDOS path, Green's function pairs through
// tbtkkpm_moments_batched and the energy sum, both with the server's table
// of max_moments rows summing the job's M terms (the same sums as a table
// of M rows).  out receives [idx][E] LDOS or [idx][E] complex G.
int rerun_fp64(tbtkkpm_server *s, const RerunJob &j, std::vector<double> &out) {
  const uint32_t E = s->E, M = j.M;
  int rc;
  Model *m = j.m;
  const size_t rd = j.kind == kLdos ? E : 2 * (size_t)E;
  out.assign(j.idx.size() * rd, 0.0);
  const int prev = swap_selected_device(s->device);
  if (j.kind == kLdos) {
    std::vector<uint32_t> miss;
    for (uint32_t k : j.idx) miss.push_back(j.sites[k]);
    rc = ldos_sites_terms(m->mat, m->table, M, miss.data(), (uint32_t)miss.size(), j.broadening,
                          TBTKKPM_FP64, out.data(), nullptr);
  } else {
    // one source per distinct from-index of the missed pairs
    std::vector<uint32_t> from, to, owner;
    std::map<uint32_t, uint32_t> src;
    for (uint32_t k : j.idx) {
      const uint32_t f = j.sites[j.pair_src[k]];
      auto it = src.find(f);
      if (it == src.end()) {
        it = src.emplace(f, (uint32_t)from.size()).first;
        from.push_back(f);
      }
      to.push_back(j.to[k]);
      owner.push_back(it->second);
    }
    std::vector<double> mu(2 * (size_t)j.idx.size() * M);
    rc = tbtkkpm_moments_batched(m->mat, from.data(), (uint32_t)from.size(), to.data(), owner.data(),
                                 (uint32_t)to.size(), M, j.broadening, TBTKKPM_FP64, mu.data(), nullptr);
    if (!rc)
      rc = energy_sum_host(m->table, mu.data(), (uint32_t)to.size(), j.kind, out.data(),
                           sizeof(double2), M);
  }
  swap_selected_device(prev);
  return rc;
}

int finish_complete(tbtkkpm_server *s, FinishBatch &fb) {
  if (fb.done.empty()) return TBTKKPM_OK;
  cudaError_t e = cudaEventSynchronize(fb.ev);
  if (e != cudaSuccess) return cuda_fail(e, "server: finish");
  const uint32_t E = s->E;
  for (size_t i = 0; i < fb.done.size(); i++) {
    Request *r = fb.done[i];
    Model *m = fb.owner[i];
    const uint32_t K = r->outputs();
    const size_t rd = r->result_doubles(E);
    const double *res = s->h_res + fb.res_off[i];
    r->ldos.assign(res, res + (size_t)K * rd);
    r->err.assign(res + (size_t)K * rd, res + (size_t)K * rd + K);
    // moment estimates -> relative errors of the LDOS or G rows
    for (uint32_t k = 0; k < K; k++)
      r->err[k] = ldos_error_estimate(r->err[k], m->table->wmax, r->ldos.data() + (size_t)k * rd, E,
                                      r->kind != kLdos);
    r->rerun.assign(K, 0);
    RerunJob j;
    for (uint32_t k = 0; k < K; k++)
      if (s->tol > 0 && !(r->err[k] <= s->tol)) j.idx.push_back(k);
    if (!j.idx.empty()) {
      j.id = r->id;
      j.m = m;
      j.kind = r->kind;
      j.M = r->M;
      j.broadening = r->broadening;
      j.sites = r->sites;
      j.to = r->to;
      j.pair_src = r->pair_src;
      fb.reruns.push_back(std::move(j));
      fb.rerun_req.push_back(r);
    }
  }
  return TBTKKPM_OK;
}

// ------------------------------------------------------------ worker

void fail_all(tbtkkpm_server *s, int rc, const std::string &msg) {
  s->failed = rc;
  s->fail_msg = msg;
  for (auto &p : s->requests) {
    Request *r = p.second.get();
    if (!r->done) {
      r->done = true;
      r->status = rc;
      r->message = msg;
    }
  }
  s->pending.clear();
  s->cv_done.notify_all();
}

// A rerun thread: FP64 recomputations of finished requests, one job at a
// time, results written back under the lock if the request still waits.
// Jobs of one model take turns on its matrix handle (its lock).
void rerun_worker(tbtkkpm_server *s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_rerun.wait(lk, [&] { return s->stop || !s->rerun_jobs.empty(); });
    if (s->stop) break;
    RerunJob j = std::move(s->rerun_jobs.front());
    s->rerun_jobs.pop_front();
    s->rerun_running += 1;
    lk.unlock();
    const auto r0 = Clock::now();
    std::vector<double> out;
    const int rc = rerun_fp64(s, j, out);
    const auto r1 = Clock::now();
    lk.lock();
    s->rerun_running -= 1;
    s->rerun_s += std::chrono::duration<double>(r1 - r0).count();
    auto it = s->requests.find(j.id);
    if (it == s->requests.end() || it->second->done) continue;  // failed or dropped meanwhile
    Request *r = it->second.get();
    if (rc) {
      r->status = rc;
      r->message = tbtkkpm_last_error();
    } else {
      const size_t rd = r->result_doubles(s->E);
      for (size_t q = 0; q < j.idx.size(); q++) {
        std::memcpy(r->ldos.data() + (size_t)j.idx[q] * rd, out.data() + q * rd, sizeof(double) * rd);
        r->rerun[j.idx[q]] = 1;
      }
      s->reruns += (double)j.idx.size();
    }
    s->latencies_ms.push_back(std::chrono::duration<double, std::milli>(r1 - r->t_submit).count());
    r->done = true;
    s->cv_done.notify_all();
  }
}

void worker(tbtkkpm_server *s) {
  cudaSetDevice(s->device);
  swap_selected_device(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  FinishBatch prev;  // launched, host half pending
  // Host half of the pending finish (lock held on entry and exit): the
  // requests complete and their waiters wake.
  auto complete_prev = [&]() -> int {
    if (prev.done.empty()) return TBTKKPM_OK;
    lk.unlock();
    const auto f0 = Clock::now();
    int rc = finish_complete(s, prev);
    const auto f1 = Clock::now();
    lk.lock();
    s->finish_s += std::chrono::duration<double>(f1 - f0).count();
    if (rc) return rc;
    // requests with FP64 recomputations complete on the rerun thread
    std::sort(prev.rerun_req.begin(), prev.rerun_req.end());
    for (Request *r : prev.done) {
      if (std::binary_search(prev.rerun_req.begin(), prev.rerun_req.end(), r)) continue;
      s->latencies_ms.push_back(std::chrono::duration<double, std::milli>(f1 - r->t_submit).count());
      r->done = true;
    }
    if (!prev.reruns.empty()) {
      for (RerunJob &j : prev.reruns) s->rerun_jobs.push_back(std::move(j));
      s->cv_rerun.notify_all();
    }
    prev.done.clear();
    prev.owner.clear();
    prev.reruns.clear();
    prev.rerun_req.clear();
    s->cv_done.notify_all();
    return TBTKKPM_OK;
  };
  int rc = TBTKKPM_OK;
  while (!s->stop) {
    bool busy = false;
    for (auto &p : s->models) busy = busy || (p->resident && p->busy);
    if (!busy && s->pending.empty()) {
      if (!prev.done.empty()) {
        if ((rc = complete_prev())) break;
        s->working = false;
        continue;
      }
      s->working = false;
      s->cv_work.wait(lk);
      continue;
    }
    const auto t0 = Clock::now();
    s->working = true;
    std::vector<MultiJoin> joins;
    std::vector<JoinRef> refs;
    std::vector<Relayout> moves;
    rc = admit(s, joins, refs, moves);
    if (!rc && !moves.empty()) {
      lk.unlock();
      rc = run_relayouts(s, moves);
      lk.lock();
      s->relayouts += (double)moves.size();
    }
    if (!rc && !joins.empty()) {
      // FP64 heads: a lane with head q starts at local step q + 1, and a
      // request ends with its last lane
      std::vector<uint32_t> head;
      lk.unlock();
      const auto j0 = Clock::now();
      rc = run_joins(s, joins, refs, head);
      const double js = std::chrono::duration<double>(Clock::now() - j0).count();
      lk.lock();
      s->join_s += js;
      s->plan_s -= js;  // plan_s counts the worker's own admission and planning
      for (size_t i = 0; !rc && i < refs.size(); i++) {
        refs[i].m->base_h[refs[i].c] -= (int32_t)head[i];
        refs[i].m->dirty = true;
      }
      for (size_t i = 0; !rc && i < refs.size(); i++) {
        Request *r = refs[i].r;
        if (r->lanes[0] != refs[i].c) continue;
        int32_t last = INT32_MIN;
        for (uint32_t c : r->lanes) last = std::max(last, refs[i].m->base_h[c]);
        r->base = last;
      }
    }
    std::vector<ClassPlan> plans;
    if (!rc) rc = plan_tick(s, plans);
    if (rc) break;
    if (plans.empty()) {
      // queued work that cannot start yet (it waits for memory)
      if ((rc = complete_prev())) break;
      s->working = false;
      s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
      continue;
    }
    // steps until the first busy request finishes, at most tick_steps
    uint32_t nsteps = s->tick_steps;
    for (auto &p : s->models) {
      Model *m = p.get();
      if (!m->resident || !m->busy) continue;
      for (uint32_t c = 0; c < m->Wmax; c++) {
        if (!m->lane_req[c]) continue;
        const Request *r = s->requests.at(m->lane_req[c]).get();
        if (r->lanes.empty() || r->lanes[0] != c) continue;  // one entry per request
        if (r->cancelled) {
          nsteps = 1;  // its lanes leave after this step
          continue;
        }
        const int64_t last = (int64_t)r->base + r->steps();  // global step of its last local step
        const int64_t left = last - (int64_t)s->n_global + 1;
        nsteps = (uint32_t)std::min<int64_t>(nsteps, std::max<int64_t>(left, 1));
      }
    }
    s->tick_no += 1;
    const auto p1 = Clock::now();
    s->plan_s += std::chrono::duration<double>(p1 - t0).count();
    lk.unlock();
    rc = run_tick(s, plans, nsteps);
    lk.lock();
    // the previous tick's requests complete while this tick runs
    const double f_before = s->finish_s;
    if (!rc) rc = complete_prev();
    const double overlap = s->finish_s - f_before;
    lk.unlock();
    cudaError_t e = cudaSuccess;
    if (!rc && (e = cudaStreamSynchronize(s->stream)) != cudaSuccess)
      rc = cuda_fail(e, "server: tick");
    if (!rc && *s->h_err)
      rc = fail(TBTKKPM_ERR_TIMEOUT, "server: a staged-row wait of a recursion step ran out");
    const double ts = std::chrono::duration<double>(Clock::now() - p1).count() - overlap;
    lk.lock();
    s->tick_s += ts;
    if (rc) break;
    s->n_global += (int32_t)nsteps;
    s->ticks += 1;
    s->steps += nsteps;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]) == cudaSuccess) s->step_s += ms * 1e-3;
    cudaGetLastError();
    for (const ClassPlan &cp : plans) s->step_bytes += cp.bytes * nsteps;
    // finished requests: every lane past its last local step; cancelled
    // ones leave their lanes now, without results
    bool cancelled = false;
    for (auto &p : s->models) {
      Model *m = p.get();
      if (!m->resident || !m->busy) continue;
      for (uint32_t c = 0; c < m->Wmax; c++) {
        const uint64_t id = m->lane_req[c];
        if (!id) continue;
        Request *r = s->requests.at(id).get();
        if (r->lanes.empty() || r->lanes[0] != c) continue;  // one entry per request
        if (r->cancelled) {
          release_request_lanes(m, r);
          r->done = true;
          r->status = TBTKKPM_ERR_CANCELLED;
          r->message = "request cancelled";
          cancelled = true;
        } else if ((int64_t)r->base + r->steps() <= (int64_t)s->n_global - 1) {
          r->finishing = true;
          prev.done.push_back(r);
          prev.owner.push_back(m);
        }
      }
    }
    if (cancelled) s->cv_done.notify_all();
    // their device half goes on the stream before any join can reuse the lanes
    lk.unlock();
    const auto f0 = Clock::now();
    rc = finish_launch(s, prev);
    const double fs = std::chrono::duration<double>(Clock::now() - f0).count();
    lk.lock();
    s->finish_s += fs;
    if (rc) break;
    for (size_t i = 0; i < prev.done.size(); i++) {
      Request *r = prev.done[i];
      release_request_lanes(prev.owner[i], r);
      s->lane_steps += (double)r->lanes.size() * r->steps();
    }
    s->busy_s += std::chrono::duration<double>(Clock::now() - t0).count();
  }
  if (rc) fail_all(s, rc, tbtkkpm_last_error());
  if (prev.ev) cudaEventDestroy(prev.ev);
  s->working = false;
}

}  // namespace
}  // namespace tbtkkpm

// ---------------------------------------------------------------- C ABI

extern "C" int tbtkkpm_server_create(uint32_t max_moments, const double *energies, uint32_t E,
                                     uint64_t hbm_budget, uint32_t tick_steps, double tolerance,
                                     tbtkkpm_server **out) {
  if (!out) return fail(TBTKKPM_ERR_ARGUMENT, "server_create: out is NULL");
  *out = nullptr;
  if (max_moments < 2) return fail(TBTKKPM_ERR_ARGUMENT, "server_create: max_moments < 2");
  if (!energies || E == 0) return fail(TBTKKPM_ERR_ARGUMENT, "server_create: empty energy grid");
  if (hbm_budget == 0) return fail(TBTKKPM_ERR_ARGUMENT, "server_create: hbm_budget is 0");
  int ndev = 0;
  tbtkkpm_device_count(&ndev);
  if (ndev == 0) return fail(TBTKKPM_ERR_CUDA, "no CUDA device available");
  auto *s = new tbtkkpm_server();
  s->device = current_device();
  s->Mmax = max_moments;
  s->ld = max_moments / 2 + 1;
  s->E = E;
  s->energies.assign(energies, energies + E);
  s->budget = hbm_budget;
  s->tick_steps = tick_steps ? tick_steps : 64;
  s->tol = tolerance;
  {
    DeviceGuard g(s->device);
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev[1]);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming);
    for (int i = 0; e == cudaSuccess && i < tbtkkpm_server::kClassStreams; i++) {
      e = cudaStreamCreateWithFlags(&s->cls_stream[i], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_join[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_err, sizeof(int));
    if (e == cudaSuccess && (s->d_err.reserve(sizeof(int)) != TBTKKPM_OK ||
                             s->d_step.reserve(sizeof(int32_t)) != TBTKKPM_OK))
      e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = cudaMemset(s->d_err.ptr, 0, sizeof(int));
    if (e != cudaSuccess) {
      s->d_err.release();
      s->d_step.release();
      if (s->h_err) cudaFreeHost(s->h_err);
      for (cudaEvent_t ev : {s->ev[0], s->ev[1], s->ev_fork})
        if (ev) cudaEventDestroy(ev);
      for (int i = 0; i < tbtkkpm_server::kClassStreams; i++) {
        if (s->ev_join[i]) cudaEventDestroy(s->ev_join[i]);
        if (s->cls_stream[i]) cudaStreamDestroy(s->cls_stream[i]);
      }
      if (s->stream) cudaStreamDestroy(s->stream);
      delete s;
      return cuda_fail(e, "server_create: stream");
    }
    *s->h_err = 0;
  }
  s->worker = std::thread(worker, s);
  for (auto &t : s->rerun_threads) t = std::thread(rerun_worker, s);
  *out = s;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_server_add_model(tbtkkpm_server *s, const uint32_t *rowptr,
                                        const uint32_t *col, const double *val, uint32_t N,
                                        double scale, uint32_t width, uint32_t *model) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_add_model: NULL server");
  if (!model) return fail(TBTKKPM_ERR_ARGUMENT, "server_add_model: model is NULL");
  if (!valid_width(width))
    return fail(TBTKKPM_ERR_ARGUMENT, "server_add_model: width %u is not a power of two in [1, %u]",
                width, kMaxWidth);
  for (uint32_t e = 0; e < s->E; e++)
    if (!(std::fabs(s->energies[e]) < scale))
      return fail(TBTKKPM_ERR_ARGUMENT,
                  "server_add_model: energy %g outside (-s, s) for s=%g", s->energies[e], scale);
  auto m = std::make_unique<Model>();
  const int prev = swap_selected_device(s->device);
  int rc = tbtkkpm_matrix_create_csr(rowptr, col, val, N, scale, &m->mat);
  tbtkkpm_table *t = nullptr;
  bool new_table = false, use_real = true, table_free = false;
  uint32_t head_steps = 0;
  if (!rc) {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->tables.find(scale);
    if (it != s->tables.end()) t = it->second;
    use_real = s->use_real;
    head_steps = s->head_steps;
    table_free = s->table_free;
  }
  if (!rc && !t) {
    rc = table_free ? tbtkkpm_table_create_clenshaw(s->Mmax, s->energies.data(), s->E, scale, &t)
                    : tbtkkpm_table_create(s->Mmax, s->energies.data(), s->E, scale, &t);
    new_table = rc == 0;
  }
  swap_selected_device(prev);
  if (rc) {
    tbtkkpm_matrix_destroy(m->mat);
    return rc;
  }
  m->N = N;
  m->W = m->Wmax = width;
  m->scale = scale;
  m->real = use_real && m->mat->values_real;
  m->head_steps = head_steps;
  m->bytes = lane_bytes(N, width, s->Mmax, s->ld, m->esize());
  if (m->bytes > s->budget) {
    tbtkkpm_matrix_destroy(m->mat);
    if (new_table) tbtkkpm_table_destroy(t);
    return fail(TBTKKPM_ERR_MEMORY,
                "server_add_model: lane memory of %llu bytes exceeds the budget of %llu",
                (unsigned long long)m->bytes, (unsigned long long)s->budget);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (new_table) {
    auto ins = s->tables.emplace(scale, t);
    if (!ins.second) tbtkkpm_table_destroy(t);  // another thread made one meanwhile
  }
  m->table = s->tables.at(scale);
  m->id = (uint32_t)s->models.size();
  *model = m->id;
  s->models.push_back(std::move(m));
  return TBTKKPM_OK;
}

namespace tbtkkpm {
namespace {

// Checks shared by both request kinds and queues the request (under s->mu).
int queue_request(tbtkkpm_server *s, std::unique_ptr<Request> r, uint64_t *request, const char *who) {
  if (s->failed) return fail(s->failed, "server: %s", s->fail_msg.c_str());
  if (r->model >= s->models.size()) return fail(TBTKKPM_ERR_ARGUMENT, "%s: no model %u", who, r->model);
  const Model *m = s->models[r->model].get();
  if (r->M < 2 || r->M > s->Mmax)
    return fail(TBTKKPM_ERR_ARGUMENT, "%s: M=%u outside [2, %u]", who, r->M, s->Mmax);
  if (!(r->broadening >= 0)) return fail(TBTKKPM_ERR_ARGUMENT, "%s: broadening < 0", who);
  for (uint32_t v : r->sites)
    if (v >= m->N) return fail(TBTKKPM_ERR_ARGUMENT, "%s: index %u >= N=%u", who, v, m->N);
  for (uint32_t v : r->to)
    if (v >= m->N) return fail(TBTKKPM_ERR_ARGUMENT, "%s: index %u >= N=%u", who, v, m->N);
  r->id = s->next_id++;
  r->t_submit = Clock::now();
  *request = r->id;
  s->pending.push_back(r->id);
  s->requests.emplace(r->id, std::move(r));
  s->cv_work.notify_one();
  return TBTKKPM_OK;
}

// Waits for a request of the given kind class and copies its results
// (shared by tbtkkpm_server_wait and tbtkkpm_server_wait_greens).
int wait_request(tbtkkpm_server *s, uint64_t request, double timeout_s, bool greens, double *out,
                 double *err_out, int32_t *rerun_out, const char *who) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "%s: NULL server", who);
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->requests.find(request);
  if (it == s->requests.end())
    return fail(TBTKKPM_ERR_ARGUMENT, "%s: no request %llu", who, (unsigned long long)request);
  Request *r = it->second.get();
  if ((r->kind != kLdos) != greens)
    return fail(TBTKKPM_ERR_ARGUMENT, "%s: request %llu is %s request", who,
                (unsigned long long)request,
                greens ? "an LDOS (tbtkkpm_server_wait)" : "a Green's-function (tbtkkpm_server_wait_greens)");
  if (!r->done && timeout_s > 0) {
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                          std::chrono::duration<double>(timeout_s));
    s->cv_done.wait_until(lk, until, [&] { return r->done; });
  }
  if (!r->done) return TBTKKPM_PENDING;
  if (r->status) {
    const int rc = fail(r->status, "server: %s", r->message.c_str());
    s->requests.erase(it);
    return rc;
  }
  const size_t K = r->outputs();
  if (out) std::memcpy(out, r->ldos.data(), sizeof(double) * K * r->result_doubles(s->E));
  if (err_out) std::memcpy(err_out, r->err.data(), sizeof(double) * K);
  if (rerun_out) std::memcpy(rerun_out, r->rerun.data(), sizeof(int32_t) * K);
  s->requests.erase(it);
  return TBTKKPM_OK;
}

}  // namespace
}  // namespace tbtkkpm

extern "C" int tbtkkpm_server_submit(tbtkkpm_server *s, uint32_t model, const uint32_t *sites,
                                     uint32_t n_sites, uint32_t M, double broadening,
                                     uint64_t *request) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_submit: NULL server");
  if (!request || (!sites && n_sites)) return fail(TBTKKPM_ERR_ARGUMENT, "server_submit: NULL pointer");
  std::lock_guard<std::mutex> lk(s->mu);
  if (model < s->models.size()) {
    const Model *m = s->models[model].get();
    if (n_sites == 0 || n_sites > m->Wmax)
      return fail(TBTKKPM_ERR_ARGUMENT, "server_submit: %u sites for a model of %u lanes", n_sites,
                  m->Wmax);
  }
  auto r = std::make_unique<Request>();
  r->model = model;
  r->sites.assign(sites, sites + n_sites);
  r->M = M;
  r->broadening = broadening;
  return queue_request(s, std::move(r), request, "server_submit");
}

extern "C" int tbtkkpm_server_submit_greens(tbtkkpm_server *s, uint32_t model, const uint32_t *to,
                                            const uint32_t *from, uint32_t n_pairs, uint32_t M,
                                            double broadening, int type, uint64_t *request) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_submit_greens: NULL server");
  if (!request || ((!to || !from) && n_pairs))
    return fail(TBTKKPM_ERR_ARGUMENT, "server_submit_greens: NULL pointer");
  if (type < TBTKKPM_ADVANCED || type > TBTKKPM_NONPRINCIPAL)
    return fail(TBTKKPM_ERR_ARGUMENT, "server_submit_greens: Unkown Green's function type %d", type);
  std::lock_guard<std::mutex> lk(s->mu);
  auto r = std::make_unique<Request>();
  r->model = model;
  r->kind = type;
  r->M = M;
  r->broadening = broadening;
  std::map<uint32_t, uint32_t> src;
  for (uint32_t k = 0; k < n_pairs; k++) {
    auto it = src.find(from[k]);
    if (it == src.end()) {
      it = src.emplace(from[k], (uint32_t)r->sites.size()).first;
      r->sites.push_back(from[k]);
    }
    r->to.push_back(to[k]);
    r->pair_src.push_back(it->second);
    r->direct = r->direct || to[k] != from[k];
  }
  if (model < s->models.size()) {
    const Model *m = s->models[model].get();
    if (n_pairs == 0 || n_pairs > m->Wmax)
      return fail(TBTKKPM_ERR_ARGUMENT, "server_submit_greens: %u pairs for a model of %u lanes",
                  n_pairs, m->Wmax);
  }
  return queue_request(s, std::move(r), request, "server_submit_greens");
}

extern "C" int tbtkkpm_server_wait(tbtkkpm_server *s, uint64_t request, double timeout_s,
                                   double *ldos_out, double *err_out, int32_t *rerun_out) {
  return wait_request(s, request, timeout_s, false, ldos_out, err_out, rerun_out, "server_wait");
}

extern "C" int tbtkkpm_server_wait_greens(tbtkkpm_server *s, uint64_t request, double timeout_s,
                                          double *G_out, double *err_out, int32_t *rerun_out) {
  return wait_request(s, request, timeout_s, true, G_out, err_out, rerun_out, "server_wait_greens");
}

extern "C" int tbtkkpm_server_cancel(tbtkkpm_server *s, uint64_t request) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_cancel: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->requests.find(request);
  if (it == s->requests.end())
    return fail(TBTKKPM_ERR_ARGUMENT, "server_cancel: no request %llu", (unsigned long long)request);
  Request *r = it->second.get();
  if (r->cancelled) return TBTKKPM_OK;
  if (r->done || r->finishing)
    return fail(TBTKKPM_ERR_STATE, "server_cancel: request %llu has finished its recursion",
                (unsigned long long)request);
  r->cancelled = true;
  auto q = std::find(s->pending.begin(), s->pending.end(), request);
  if (q != s->pending.end()) {
    // still queued: it never takes lanes
    s->pending.erase(q);
    r->done = true;
    r->status = TBTKKPM_ERR_CANCELLED;
    r->message = "request cancelled";
    s->cv_done.notify_all();
  }
  // in flight: the worker frees its lanes at the next step boundary
  s->cv_work.notify_one();
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_server_stats(tbtkkpm_server *s, double *out, uint32_t n) {
  if (!s || (!out && n)) return fail(TBTKKPM_ERR_ARGUMENT, "server_stats: NULL pointer");
  std::lock_guard<std::mutex> lk(s->mu);
  double v[TBTKKPM_STAT_COUNT] = {0};
  std::vector<double> l = s->latencies_ms;
  v[TBTKKPM_STAT_COMPLETED] = (double)l.size();
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) {
      const size_t i = (size_t)std::min<double>(l.size() - 1, std::ceil(p * l.size()) - 1);
      return l[i];
    };
    v[TBTKKPM_STAT_P50_MS] = pct(0.50);
    v[TBTKKPM_STAT_P99_MS] = pct(0.99);
    double sum = 0;
    for (double x : l) sum += x;
    v[TBTKKPM_STAT_MEAN_MS] = sum / l.size();
  }
  v[TBTKKPM_STAT_RERUNS] = s->reruns;
  v[TBTKKPM_STAT_TICKS] = s->ticks;
  v[TBTKKPM_STAT_STEPS] = s->steps;
  v[TBTKKPM_STAT_LANE_STEPS] = s->lane_steps;
  v[TBTKKPM_STAT_RESIDENT] = (double)s->resident;
  v[TBTKKPM_STAT_EVICTIONS] = s->evictions;
  v[TBTKKPM_STAT_WAITED] = s->waited;
  v[TBTKKPM_STAT_BUSY_S] = s->busy_s;
  v[TBTKKPM_STAT_STEP_S] = s->step_s;
  v[TBTKKPM_STAT_STEP_BYTES] = s->step_bytes;
  v[TBTKKPM_STAT_FINISH_S] = s->finish_s;
  v[TBTKKPM_STAT_RERUN_S] = s->rerun_s;
  v[TBTKKPM_STAT_JOIN_S] = s->join_s;
  v[TBTKKPM_STAT_PLAN_S] = s->plan_s;
  v[TBTKKPM_STAT_TICK_S] = s->tick_s;
  v[TBTKKPM_STAT_GRAPH_TICKS] = s->graph_ticks;
  v[TBTKKPM_STAT_RELAYOUTS] = s->relayouts;
  for (uint32_t i = 0; i < n && i < TBTKKPM_STAT_COUNT; i++) out[i] = v[i];
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_server_set_config(tbtkkpm_server *s, uint32_t width, int tpr, int vpt,
                                         int minb) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_set_config: NULL server");
  const bool cplx = find_multi(tpr, vpt, minb, false) != nullptr;
  const bool real = find_multi(tpr, vpt, minb, true) != nullptr;
  if (!valid_width(width) || tpr * vpt != (int)width || !(cplx || real))
    return fail(TBTKKPM_ERR_UNSUPPORTED,
                "server_set_config: no compiled step (tpr=%d, vpt=%d, minb=%d) for width %u", tpr,
                vpt, minb, width);
  std::lock_guard<std::mutex> lk(s->mu);
  // the lane class(es) this shape is compiled for
  if (cplx) s->config[width] = {tpr, vpt, minb};
  if (real) s->config[width | 1u << 16] = {tpr, vpt, minb};
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_server_step_configs(int real, uint32_t width, int *out, int cap) {
  if (cap > 0 && !out) return fail(TBTKKPM_ERR_ARGUMENT, "server_step_configs: NULL out");
  int n = 0;
  for (const MultiEntry *e : multi_entries(real != 0)) {
    if ((uint32_t)(e->tpr * e->vpt) != width) continue;
    if (n < cap) {
      out[3 * n] = e->tpr;
      out[3 * n + 1] = e->vpt;
      out[3 * n + 2] = e->minb;
    }
    n++;
  }
  return n;
}

extern "C" int tbtkkpm_server_set_table_free(tbtkkpm_server *s, int enable) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_set_table_free: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->table_free = enable != 0;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_server_set_fp64_head(tbtkkpm_server *s, uint32_t steps) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_set_fp64_head: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->head_steps = steps;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_server_set_graphs(tbtkkpm_server *s, int enable) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_set_graphs: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->use_graphs = enable != 0;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_server_set_adaptive_width(tbtkkpm_server *s, int enable) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_set_adaptive_width: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->adaptive_width = enable != 0;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_server_set_wait_limit(tbtkkpm_server *s, uint32_t polls) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_set_wait_limit: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->wait_limit = polls == TBTKKPM_WAIT_DEFAULT ? kWaitLimit : polls;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_server_set_real(tbtkkpm_server *s, int enable) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_set_real: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->use_real = enable != 0;
  return TBTKKPM_OK;
}

namespace tbtkkpm {
namespace {

// Times every compiled configuration of the probe model's lane class
// (under s->mu, server idle) and keeps the fastest for that class.
int tune_class(tbtkkpm_server *s, Model *probe, uint32_t width, uint32_t probe_steps,
               const MultiEntry **best_out, double *best_ms_out) {
  DeviceGuard g(s->device);
  cudaStream_t st = s->stream;
  // a private copy of the lane state: every lane busy from global step 1
  const uint32_t W = width, N = probe->N, Mp = 2 * probe_steps + 2, ldp = Mp / 2 + 1;
  const bool real = probe->real;  // the class of the probe model is tuned
  const size_t es = probe->esize();
  DevBuf vec[2], dots, mu, mud, base, laneM, bitmap, tlist, dm, dh, tmap, tdesc, truns;
  int rc;
  if ((rc = vec[0].reserve(es * (size_t)N * W)) ||
      (rc = vec[1].reserve(es * (size_t)N * W)) ||
      (rc = dots.reserve(2 * sizeof(long long) * W)) || (rc = mu.reserve(sizeof(double2) * W * Mp)) ||
      (rc = mud.reserve(sizeof(double2) * W * ldp)) || (rc = base.reserve(4 * W)) ||
      (rc = laneM.reserve(4 * W)) || (rc = bitmap.reserve(4 * (size_t)((N + 31) / 32))) ||
      (rc = tlist.reserve(8 * W)) || (rc = dm.reserve(sizeof(MultiModel))) ||
      (rc = dh.reserve(sizeof(MultiHeader))))
    return rc;
  std::vector<int32_t> base_h(W, 0);
  std::vector<uint32_t> M_h(W, Mp), bm((N + 31) / 32, 0), tl(2 * (size_t)W);
  std::vector<std::pair<uint32_t, uint32_t>> t;
  std::vector<MultiJoin> joins;
  for (uint32_t c = 0; c < W; c++) {
    const uint32_t site = (uint32_t)((uint64_t)c * N / W);
    t.push_back({site, c});
    bm[site >> 5] |= 1u << (site & 31);
    joins.push_back({vec[0].as<float2>(), mu.as<double2>() + (size_t)c * Mp,
                     mud.as<double2>() + (size_t)c * ldp, N, c, site, W, real ? 1u : 0u});
  }
  std::sort(t.begin(), t.end());
  for (uint32_t i = 0; i < W; i++) {
    tl[i] = t[i].first;
    tl[W + i] = t[i].second;
  }
  cudaError_t e;
  DevBuf dj;
  if ((rc = dj.reserve(sizeof(MultiJoin) * W))) return rc;
  if ((e = cudaMemsetAsync(vec[1].ptr, 0, es * (size_t)N * W, st)) ||
      (e = cudaMemsetAsync(dots.ptr, 0, 2 * sizeof(long long) * W, st)) ||
      (e = cudaMemcpyAsync(base.ptr, base_h.data(), 4 * W, cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(laneM.ptr, M_h.data(), 4 * W, cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(bitmap.ptr, bm.data(), 4 * bm.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(tlist.ptr, tl.data(), 4 * tl.size(), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(dj.ptr, joins.data(), sizeof(MultiJoin) * W, cudaMemcpyHostToDevice, st)))
    return cuda_fail(e, "server_autotune: staging");
  kpm_multi_join<<<dim3(std::max(1u, std::min(blocks_for(std::max(N, Mp)), 512u)), W), 256, 0, st>>>(
      dj.as<MultiJoin>(), Mp, ldp);
  count_launches(1);
  cudaEvent_t ev[2];
  cudaEventCreate(&ev[0]);
  cudaEventCreate(&ev[1]);
  const MultiEntry *best = nullptr;
  double best_ms = 0;
  int32_t n = 1;
  for (const MultiEntry *ep : multi_entries(real)) {
    if (rc) break;
    const MultiEntry &en = *ep;
    if ((uint32_t)(en.tpr * en.vpt) != W) continue;
    // a tile-staged entry needs the probe's plan and a ring that fits
    const TilePlan *plan = model_plan(probe, W, &en, &rc);
    if (rc) break;
    TiledLayout ly{};
    if (is_multi_tiled(en.minb)) {
      if (!plan) continue;
      ly = multi_layout(&en, W, real, plan->wmax, plan->umax);
      if (ly.stages == 0) continue;
    }
    MultiModel d{};
    d.A.slice_ptr = probe->mat->slice_ptr.as<uint32_t>();
    d.A.col = probe->mat->scol.as<uint32_t>();
    d.A.val = probe->mat->sval.as<double2>();
    d.A.vre = real ? probe->mat->sreal.as<double>() : nullptr;
    d.A.N = N;
    d.A.nslices = probe->mat->nslices;
    d.vec[0] = vec[0].as<float2>();
    d.vec[1] = vec[1].as<float2>();
    d.bitmap = bitmap.as<uint32_t>();
    d.trow = tlist.as<uint32_t>();
    d.tcol = tlist.as<uint32_t>() + W;
    d.tcount = W;
    d.base = base.as<int32_t>();
    d.lane_M = laneM.as<uint32_t>();
    d.dots = dots.as<long long>();
    d.mu = mu.as<double2>();
    d.mu_direct = mud.as<double2>();
    d.tile0 = 0;
    d.ntiles = plan ? plan->ntiles
                    : (uint32_t)(((uint64_t)d.A.nslices * 32 + kBlock / en.tpr - 1) / (kBlock / en.tpr));
    if (plan) {
      d.p_hdr = plan->hdr;
      d.p_runs = plan->runs;
      d.p_slot = plan->eslot;
      d.p_val = plan->eval;
      d.p_nruns = plan->nruns;
      d.run0 = 0;
    }
    // one model: every tile maps to model 0
    if ((rc = tmap.reserve(4 * (size_t)d.ntiles)) ||
        (rc = tdesc.reserve(16 * kDescWords * (size_t)d.ntiles)) ||
        (rc = truns.reserve(8 * (size_t)std::max(d.p_nruns, 1u))))
      break;
    uint32_t run = kRun;
    if (plan) {
      const uint32_t grid = (uint32_t)multi_tiled_bps(en.minb) * (uint32_t)sm_count(s->device);
      run = std::max(kRun, std::min(32u, d.ntiles / std::max(4 * grid, 1u)));
    }
    MultiHeader h{1, d.ntiles, n, tmap.as<uint32_t>(), tdesc.as<uint4>(), truns.as<uint2>(), run};
    // parity of the buffers follows the global step, so the probe keeps
    // counting across configurations
    if ((e = cudaMemcpyAsync(dm.ptr, &d, sizeof(d), cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(dh.ptr, &h, sizeof(h), cudaMemcpyHostToDevice, st))) {
      rc = cuda_fail(e, "server_autotune: descriptors");
      break;
    }
    if (plan) {
      kpm_multi_tilemap_tiled<<<1, 256, 0, st>>>(dm.as<MultiModel>(), dh.as<MultiHeader>(),
                                                 (uint32_t)multi_tiled_rows(en.minb), tdesc.as<uint4>(),
                                                 truns.as<uint2>());
      count_launches(1);
    } else if ((e = cudaMemsetAsync(tmap.ptr, 0, 4 * (size_t)d.ntiles, st))) {
      rc = cuda_fail(e, "server_autotune: tile map");
      break;
    }
    const MultiLaunch ml{ly, s->d_err.as<int>(), kWaitLimit};
    for (uint32_t k = 0; k < probe_steps; k++) {
      if (k == 1) cudaEventRecord(ev[0], st);
      en.launch(st, s->device, dm.as<MultiModel>(), dh.as<MultiHeader>(), k, W, ldp, ml);
      kpm_multi_finalize<<<1, std::min<uint32_t>(std::max(W, 32u), 64u), 0, st>>>(
          dm.as<MultiModel>(), dh.as<MultiHeader>(), k, W, Mp, ldp);
    }
    count_launches(2ull * probe_steps);
    cudaEventRecord(ev[1], st);
    if ((e = cudaEventSynchronize(ev[1])) != cudaSuccess) {
      rc = cuda_fail(e, "server_autotune: probe");
      break;
    }
    int werr = 0;
    if ((e = cudaMemcpy(&werr, s->d_err.ptr, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) {
      rc = cuda_fail(e, "server_autotune: probe");
      break;
    }
    if (werr) {
      rc = fail(TBTKKPM_ERR_TIMEOUT, "server_autotune: a staged-row wait ran out");
      break;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    const double per = ms / (probe_steps - 1);
    if (!best || per < best_ms) {
      best = &en;
      best_ms = per;
    }
    n += (int32_t)probe_steps;
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  cudaStreamSynchronize(st);
  if (rc) return rc;
  if (!best) return fail(TBTKKPM_ERR_UNSUPPORTED, "server_autotune: no kernel for width %u", W);
  s->config[W | (real ? 1u << 16 : 0u)] = {best->tpr, best->vpt, best->minb};
  s->tuned.insert(W | (real ? 1u << 16 : 0u));
  // a tile-staged pick: the plans of every model of the class now, not in
  // the first tick that needs them
  for (auto &p : s->models) {
    if (p->Wmax < W || (!s->adaptive_width && p->Wmax != W) || p->real != real) continue;
    model_plan(p.get(), W, best, &rc);
    if (rc) return rc;
  }
  *best_out = best;
  *best_ms_out = best_ms;
  return TBTKKPM_OK;
}

}  // namespace
}  // namespace tbtkkpm

extern "C" int tbtkkpm_server_autotune(tbtkkpm_server *s, uint32_t width, uint32_t probe_steps,
                                       int *tpr, int *vpt, int *minb, double *ms_per_step) {
  if (!s) return fail(TBTKKPM_ERR_ARGUMENT, "server_autotune: NULL server");
  if (!valid_width(width)) return fail(TBTKKPM_ERR_ARGUMENT, "server_autotune: bad width %u", width);
  if (probe_steps < 2) return fail(TBTKKPM_ERR_ARGUMENT, "server_autotune: probe_steps < 2");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->failed) return fail(s->failed, "server: %s", s->fail_msg.c_str());
  if (s->working || !s->pending.empty() || !s->rerun_jobs.empty() || s->rerun_running)
    return fail(TBTKKPM_ERR_STATE, "server_autotune: the server is busy");
  for (auto &p : s->models)
    if (p->busy) return fail(TBTKKPM_ERR_STATE, "server_autotune: the server is busy");
  // the largest model of each lane class (real, complex) of this width
  Model *probe[2] = {nullptr, nullptr};
  for (auto &p : s->models) {
    Model *&q = probe[p->real ? 1 : 0];
    if (p->Wmax == width && (!q || p->N > q->N)) q = p.get();
  }
  if (!probe[0] && !probe[1]) return fail(TBTKKPM_ERR_STATE, "server_autotune: no model of width %u", width);
  const int main = !probe[0] || (probe[1] && probe[1]->N > probe[0]->N) ? 1 : 0;
  const MultiEntry *best[2] = {nullptr, nullptr};
  double best_ms[2] = {0, 0};
  for (int c = 0; c < 2; c++) {
    if (!probe[c]) continue;
    const int rc = tune_class(s, probe[c], width, probe_steps, &best[c], &best_ms[c]);
    if (rc) return rc;
    // the narrower widths these models step at when few lanes are busy
    // (once: another width's autotune may have measured them)
    for (uint32_t w = width / 2; s->adaptive_width && w >= std::min(kMinStepWidth, width); w /= 2) {
      if (s->tuned.count(w | (probe[c]->real ? 1u << 16 : 0u))) continue;
      const MultiEntry *b = nullptr;
      double ms = 0;
      const int rn = tune_class(s, probe[c], w, probe_steps, &b, &ms);
      if (rn) return rn;
    }
  }
  if (tpr) *tpr = best[main]->tpr;
  if (vpt) *vpt = best[main]->vpt;
  if (minb) *minb = best[main]->minb;
  if (ms_per_step) *ms_per_step = best_ms[main];
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_server_destroy(tbtkkpm_server *s) {
  if (!s) return TBTKKPM_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->cv_rerun.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (auto &t : s->rerun_threads)
    if (t.joinable()) t.join();
  {
    DeviceGuard g(s->device);
    cudaStreamSynchronize(s->stream);
    for (auto &p : s->models) {
      p->release_lanes();
      tbtkkpm_matrix_destroy(p->mat);
    }
    for (auto &t : s->tables) tbtkkpm_table_destroy(t.second);
    for (DevBuf *b : {&s->d_models, &s->d_hdr, &s->d_joins, &s->d_done, &s->d_pairs, &s->d_stage,
                      &s->d_damp, &s->d_tiles, &s->d_tdesc, &s->d_truns, &s->d_err, &s->d_step})
      b->release();
    s->head_ws.release();
    s->d_res.release();
    if (s->h_res) cudaFreeHost(s->h_res);
    if (s->h_err) cudaFreeHost(s->h_err);
    for (cudaEvent_t &ev : s->ev)
      if (ev) cudaEventDestroy(ev);
    if (s->tick_exec) cudaGraphExecDestroy(s->tick_exec);
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    for (int i = 0; i < tbtkkpm_server::kClassStreams; i++) {
      if (s->ev_join[i]) cudaEventDestroy(s->ev_join[i]);
      if (s->cls_stream[i]) cudaStreamDestroy(s->cls_stream[i]);
    }
    cudaStreamDestroy(s->stream);
  }
  delete s;
  return TBTKKPM_OK;
}
