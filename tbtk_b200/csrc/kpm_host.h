// Host-side objects behind the opaque handles of include/tbtkkpm.h.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstddef>
#include <cstdint>
#include <map>
#include <mutex>

namespace tbtkkpm {

int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
int current_device();
// Sets the device handle creations on this thread use (-1: the CUDA current
// device) and returns the previous selection.
int swap_selected_device(int device);
void count_launches(uint64_t n);
int sm_count(int device);

// CUDA events around the phases of one call on a handle's stream.
struct PhaseTimer {
  bool enabled = false;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  bool pending = false;
  double recursion_ms = 0, energy_ms = 0;
  uint64_t step_launches = 0, pending_steps = 0;
  int enable(bool on);
  void mark(cudaStream_t st, int i) {
    if (enabled) cudaEventRecord(ev[i], st);
  }
  // After the stream reached ev[3]: adds ev0->ev1 to the recursion time and
  // ev2->ev3 to the energy-sum time.
  void collect();
  void destroy();
};

// A grow-only device allocation.
struct DevBuf {
  void *ptr = nullptr;
  size_t cap = 0;
  int reserve(size_t n);
  void release();
  template <typename T> T *as() const { return static_cast<T *>(ptr); }
};

// Makes `dev` current for the scope and restores the previous device.
struct DeviceGuard {
  int prev = 0, target = 0;
  explicit DeviceGuard(int dev);
  ~DeviceGuard();
};

// Per-call workspace of a matrix handle, reused across calls.
struct Workspace {
  DevBuf vec[2];      // two [N][Bp] vector buffers
  DevBuf bitmap;      // ceil(N/32) words
  DevBuf tgt;         // target rows, columns, output slots (3*T uint32)
  DevBuf from;        // source rows
  DevBuf mu;          // [K][M] complex moments
  DevBuf damp;        // [M] damping numerators
  DevBuf out;         // results ([B][E] LDOS)
  DevBuf mu_direct;   // [K][steps+1] directly gathered moments (doubling runs)
  DevBuf dots;        // [grid][2][Bp] per-block dot products (doubling runs)
  DevBuf col_out;     // [Bp] output slot of each batch column (doubling runs)
  DevBuf err;         // device flag of a bounded wait that ran out
  DevBuf head, head_jobs, head_res;  // FP64 head of doubling runs (scratch, jobs, results)
  void release() {
    for (DevBuf *b : {&vec[0], &vec[1], &bitmap, &tgt, &from, &mu, &damp, &out, &mu_direct,
                      &dots, &col_out, &err, &head, &head_jobs, &head_res})
      b->release();
  }
};

// Per-tile gather plan of a matrix for tiles of R consecutive rows, read
// by the tile-staged steps (kpm_tiled.cuh).
struct TilePlan {
  const uint4 *hdr;        // [ntiles] {ent_begin, run_begin, nuniq, w | nruns << 16}
  const uint2 *runs;       // {first column, slot_start << 16 | length}
  const uint16_t *eslot;   // [chunks][R] shared-memory slot of each entry's column
  const void *eval;        // [chunks][R] value (double for real, double2 for complex)
  uint32_t N, ntiles, R;
  uint32_t umax, wmax;     // most distinct outside columns / entries per row of a tile
  uint32_t nruns;          // runs of all tiles
  uint32_t pairs;          // row-pair plan: entries of [w][R/2] row pairs, two values each
};

// Byte layout of one shared-memory ring stage of a tile-staged step
// (offsets from the stage start) and the ring.
struct TiledLayout {
  uint32_t stages, stage_bytes, off_slots, off_xs, off_prev;
};

// A plan and its device arrays; ok is false when some tile has more entries
// than the builder sorts in shared memory.
struct TilePlanStore {
  bool ok = false;
  TilePlan plan{};
  DevBuf hdr, runs, eslot, eval;
  void release() {
    hdr.release();
    runs.release();
    eslot.release();
    eval.release();
  }
};

}  // namespace tbtkkpm

struct tbtkkpm_matrix {
  int device = 0;
  cudaStream_t stream = nullptr;      // the stream work is issued on
  cudaStream_t own_stream = nullptr;  // created with the handle
  uint32_t N = 0;
  uint64_t nnz = 0;
  double scale = 1;
  tbtkkpm::DevBuf rowptr, col, val2;  // CSR of 2H/s (complex128)
  // SELL-32 copy the recursion reads: slice_ptr[nslices+1] (chunk offsets),
  // scol/sval[chunks*32]
  tbtkkpm::DevBuf slice_ptr, scol, sval;
  // real matrix (every scaled value has a zero imaginary part): the real
  // parts in SELL order, read by the real-vector steps of the mixed path
  bool values_real = false;
  bool use_real = true;  // tbtkkpm_matrix_set_real
  tbtkkpm::DevBuf sreal;
  // structurally symmetric pattern: doubling runs may take their first
  // head_steps steps in FP64 on the rows those steps reach
  bool pattern_symmetric = false;
  uint32_t head_steps = 32;  // tbtkkpm_matrix_set_fp64_head (kPrefixSteps)
  // tbtkkpm_matrix_set_wait_limit: polls per staged-row wait of the
  // tile-staged steps (TBTKKPM_WAIT_DEFAULT: the library's bound)
  uint32_t wait_limit = 0xffffffffu;
  // tbtkkpm_matrix_set_batch_width: sources per recursion batch, per
  // precision (0: the library's choice, batch_width_for in recursion.cu)
  uint32_t batch_width[3] = {0, 0, 0};
  uint32_t nslices = 0;
  uint64_t chunks = 0;
  tbtkkpm::Workspace ws;
  tbtkkpm::PhaseTimer timer;
  // autotuned step configuration per (kernel class, padded batch width):
  // {threads per row, values per thread, min blocks per SM}
  std::map<uint64_t, std::array<int, 3>> tuned;
  // tile plans by (rows per tile, complex values, row pairs): key
  // 1024*pairs + 2*R + complex
  std::map<int, tbtkkpm::TilePlanStore> plans;
  std::mutex lock;
  void release_all() {
    for (auto &p : plans) p.second.release();
    plans.clear();
    rowptr.release();
    col.release();
    val2.release();
    slice_ptr.release();
    scol.release();
    sval.release();
    sreal.release();
    ws.release();
    timer.destroy();
  }
};

struct tbtkkpm_table {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t M = 0, E = 0;
  // table-free handle (tbtkkpm_table_create_clenshaw): energies and scale
  // only, the energy sums run Clenshaw recurrences (kpm_clenshaw)
  bool clenshaw = false;
  // Chebyshev-node grid handle (tbtkkpm_table_create_chebyshev): the
  // energy sums run one FFT per vector (kpm_chebyshev_grid) over `twiddle`,
  // [2E] complex e^{i pi m / (2E)}
  bool chebyshev_grid = false;
  double scale = 0;
  // error weight of this grid: the largest weight of the energy sum,
  // max_e |T[1][e]| / pi = max_e 2 / (pi s sqrt(1 - (E_e/s)^2)), times the
  // grid's edge coherence (edge_coherence, recursion.cu): the scale that
  // turns a moment error into an LDOS error (ldos_error_estimate)
  double wmax = 0;
  tbtkkpm::DevBuf energies;  // [E]
  tbtkkpm::DevBuf twiddle;   // [2E] complex128 (Chebyshev-node grid)
  tbtkkpm::DevBuf table;   // [M][E] complex128
  tbtkkpm::DevBuf mu, out; // staging for energy sums
  std::mutex lock;
};

#include <vector>

namespace tbtkkpm {

// Energy sum of `type` (0-3 Green's functions, 4 = LDOS) over K moment
// vectors [K][terms] on the device (terms 0: the table's M).
int launch_energy_sum(cudaStream_t st, const tbtkkpm_table *t, const double2 *mu, uint32_t K,
                      int type, void *out, uint32_t terms = 0);
// Energy sum of host moments [K][terms] into host `out` (terms 0: the
// table's M; out_elem the bytes of one result value).
int energy_sum_host(tbtkkpm_table *t, const double *mu, uint32_t K, int type, void *out,
                    size_t out_elem, uint32_t terms);
// tbtkkpm_ldos_sites for M <= the table's rows moments.
int ldos_sites_terms(tbtkkpm_matrix *m, tbtkkpm_table *t, uint32_t M, const uint32_t *sites,
                     uint32_t B, double broadening, int precision, double *ldos_out,
                     double *err_out);
// Lorentz damping numerators a[n] and denominator b (host libm).
void damping_factors(uint32_t M, double broadening, std::vector<double> &a, double &b);
// Error estimate of doubled moments against the directly gathered ones.
// Error weight of a grid (tbtkkpm_table::wmax): its largest energy-sum
// weight times edge_coherence of its smallest node angle acos|E/s|.
double grid_weight_max(const double *energies, uint32_t E, double scale);
double edge_coherence(double theta_min);
// LDOS-space error estimate of a doubling run from its moment estimate
// (doubling_error): moment_err * wmax / max_e |v_e| over the result row, v
// the LDOS (complex false), or G / pi for a Green's function row (complex
// true, E interleaved pairs).  0 when the row is zero.
double ldos_error_estimate(double moment_err, double wmax, const double *row, uint32_t E, bool complex);
void doubling_error(const std::vector<double2> &mu, const std::vector<double2> &direct,
                    uint32_t K, uint32_t M, uint32_t ld, double *err);
// The matrix's gather plan for R-row tiles (real or complex values; pairs:
// the row-pair plan of complex values, R >= 16), built on first use; *out is
// null when some tile is too large for the builder.
int tile_plan(tbtkkpm_matrix *m, int R, bool cplx, const TilePlan **out, bool pairs = false);

}  // namespace tbtkkpm
