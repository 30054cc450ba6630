// C ABI of the KPM path (include/tbtkkpm.h): handles, workspace, dispatch.
#include "tbtkkpm.h"
#include "kpm_kernels.cuh"
#include "kpm_prefix.cuh"
#include "kpm_host.h"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace tbtkkpm {

// ---------------------------------------------------------------- errors

static thread_local std::string g_error;
static thread_local int g_device = -1;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation)
    return fail(TBTKKPM_ERR_MEMORY, "%s: %s", what, cudaGetErrorString(e));
  return fail(TBTKKPM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int current_device() {
  if (g_device >= 0) return g_device;
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

int swap_selected_device(int device) {
  const int prev = g_device;
  g_device = device;
  return prev;
}

int sm_count(int device) {
  static std::atomic<int> cache[64];
  if (device < 0 || device >= 64) return 148;
  int v = cache[device].load();
  if (v == 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0) {
      cudaGetLastError();
      v = 148;
    }
    cache[device].store(v);
  }
  return v;
}

static std::atomic<uint64_t> g_launches{0};

void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ---------------------------------------------------------------- phase timer

int PhaseTimer::enable(bool on) {
  if (on && !ev[0]) {
    for (auto &e : ev) {
      cudaError_t r = cudaEventCreate(&e);
      if (r != cudaSuccess) return cuda_fail(r, "cudaEventCreate");
    }
  }
  enabled = on;
  return TBTKKPM_OK;
}

void PhaseTimer::collect() {
  if (!enabled || !pending) return;
  float a = 0, b = 0;
  if (cudaEventElapsedTime(&a, ev[0], ev[1]) == cudaSuccess) recursion_ms += a;
  if (cudaEventElapsedTime(&b, ev[2], ev[3]) == cudaSuccess) energy_ms += b;
  cudaGetLastError();
  step_launches += pending_steps;
  pending_steps = 0;
  pending = false;
}

void PhaseTimer::destroy() {
  for (auto &e : ev)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  enabled = false;
}

// ---------------------------------------------------------------- buffers

int DevBuf::reserve(size_t n) {
  if (n <= cap) return TBTKKPM_OK;
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc(&ptr, n);
  if (e != cudaSuccess) {
    ptr = nullptr;
    return cuda_fail(e, "cudaMalloc (workspace)");
  }
  cap = n;
  return TBTKKPM_OK;
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  cap = 0;
}

DeviceGuard::DeviceGuard(int dev) {
  cudaGetDevice(&prev);
  if (prev != dev) cudaSetDevice(dev);
  target = dev;
}
DeviceGuard::~DeviceGuard() {
  if (prev != target) cudaSetDevice(prev);
}

// ---------------------------------------------------------------- matrix build kernels

// val2 = (v * complex(1/s, 0)) * complex(2, 0), each complex product in the
// reference's operation order (ChebyshevExpander.cpp:147,168 through
// SparseMatrix::operator*=, SparseMatrix.h:1106-1127).
__global__ void k_scale_values(uint64_t nnz, double inv, double2 *val) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz) return;
  double2 v = cmul_exact(val[i], make_double2(inv, 0.0));
  val[i] = cmul_exact(v, make_double2(2.0, 0.0));
}

// Triplet builder: keys sorted by (row, col) with the insertion order kept
// among equal keys (stable radix sort), then each run of equal keys is folded
// from the back, d0 + (d1 + (d2 + ...)) (SparseMatrix::mergeLIL,
// SparseMatrix.h:1393-1414).
__global__ void k_mark_heads(uint64_t n, const uint64_t *keys, uint32_t *head) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void k_fold_runs(uint64_t n, const uint64_t *keys, const uint64_t *order,
                            const double2 *vals_in, const uint32_t *head,
                            const uint32_t *pos, uint32_t *col, double2 *val,
                            uint32_t *row_of) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !head[i]) return;
  uint64_t e = i;
  while (e + 1 < n && keys[e + 1] == keys[i]) e++;
  double2 acc = vals_in[order[e]];
  for (uint64_t y = e; y > i; y--) acc = cadd_exact(vals_in[order[y - 1]], acc);
  const uint32_t o = pos[i];
  col[o] = (uint32_t)(keys[i] & 0xffffffffu);
  val[o] = acc;
  row_of[o] = (uint32_t)(keys[i] >> 32);
}

// rowptr[r] = first merged entry with row >= r.
__global__ void k_rowptr(uint64_t nnz, uint32_t N, const uint32_t *row_of, uint32_t *rowptr) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nnz) return;
  const uint32_t lo = (i == 0) ? 0u : row_of[i - 1] + 1;
  const uint32_t hi = (i == nnz) ? N : row_of[i];
  for (uint32_t r = lo; r <= hi && r <= N; r++) rowptr[r] = (uint32_t)i;
}

__global__ void k_make_keys(uint64_t n, const uint32_t *rows, const uint32_t *cols,
                            uint64_t *keys, uint64_t *order) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = ((uint64_t)rows[i] << 32) | cols[i];
  order[i] = i;
}

static inline unsigned blocks_for(uint64_t n, unsigned bs = 256) {
  return (unsigned)((n + bs - 1) / bs);
}

// SELL-32 copy of the scaled CSR (the layout the recursion reads).
static int build_sell(tbtkkpm_matrix *m, cudaStream_t st) {
  const uint32_t N = m->N;
  const uint32_t ns = (N + 31) / 32;
  m->nslices = ns;
  DevBuf width, tmp;
  int rc;
  if ((rc = width.reserve(4 * ((size_t)ns + 1))) ||
      (rc = m->slice_ptr.reserve(4 * ((size_t)ns + 1))))
    return rc;
  cudaError_t e = cudaMemsetAsync(width.ptr, 0, 4 * ((size_t)ns + 1), st);
  if (e != cudaSuccess) return cuda_fail(e, "SELL build");
  k_sell_width<<<blocks_for(ns), 256, 0, st>>>(N, ns, m->rowptr.as<uint32_t>(),
                                               width.as<uint32_t>());
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, width.as<uint32_t>(), m->slice_ptr.as<uint32_t>(),
                                (int64_t)ns + 1, st);
  if ((rc = tmp.reserve(std::max<size_t>(tb, 16)))) return rc;
  cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, width.as<uint32_t>(), m->slice_ptr.as<uint32_t>(),
                                (int64_t)ns + 1, st);
  uint32_t chunks = 0;
  e = cudaMemcpyAsync(&chunks, m->slice_ptr.as<uint32_t>() + ns, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  width.release();
  tmp.release();
  if (e != cudaSuccess) return cuda_fail(e, "SELL build");
  m->chunks = chunks;
  const size_t slots = std::max<size_t>((size_t)chunks * 32, 1);
  if ((rc = m->scol.reserve(4 * slots)) || (rc = m->sval.reserve(16 * slots))) return rc;
  k_sell_fill<<<blocks_for((uint64_t)ns * 32), 256, 0, st>>>(
      N, ns, m->rowptr.as<uint32_t>(), m->col.as<uint32_t>(), m->val2.as<double2>(),
      m->slice_ptr.as<uint32_t>(), m->scol.as<uint32_t>(), m->sval.as<double2>());
  count_launches(2);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "SELL build");
  // real parts for the real-vector steps, kept only for a real matrix
  DevBuf flag;
  if ((rc = m->sreal.reserve(8 * slots)) || (rc = flag.reserve(4))) return rc;
  unsigned complex_flag = 0;
  if ((e = cudaMemsetAsync(flag.ptr, 0, 4, st)) != cudaSuccess) return cuda_fail(e, "SELL build");
  k_sell_real<<<blocks_for(slots), 256, 0, st>>>(slots, m->sval.as<double2>(), m->sreal.as<double>(),
                                                flag.as<unsigned>());
  count_launches(1);
  e = cudaMemcpyAsync(&complex_flag, flag.ptr, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "SELL build");
  m->values_real = complex_flag == 0;
  if (!m->values_real) m->sreal.release();
  // structural symmetry, which the FP64 head of doubling runs needs
  unsigned asym = 0;
  if (N > 0) {
    if ((e = cudaMemsetAsync(flag.ptr, 0, 4, st)) != cudaSuccess) return cuda_fail(e, "SELL build");
    k_pattern_check<<<blocks_for(N), 256, 0, st>>>(N, m->rowptr.as<uint32_t>(), m->col.as<uint32_t>(),
                                                   flag.as<unsigned>());
    count_launches(1);
    e = cudaMemcpyAsync(&asym, flag.ptr, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "SELL build");
  }
  m->pattern_symmetric = N > 0 && asym == 0;
  return TBTKKPM_OK;
}

}  // namespace tbtkkpm

using namespace tbtkkpm;

// ---------------------------------------------------------------- C ABI: misc

extern "C" const char *tbtkkpm_last_error(void) { return g_error.c_str(); }

extern "C" int tbtkkpm_version(void) { return 10000; }

extern "C" uint64_t tbtkkpm_kernel_launches(void) { return g_launches.load(); }

extern "C" int tbtkkpm_matrix_set_profiling(tbtkkpm_matrix *m, int enable) {
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_set_profiling: NULL handle");
  std::lock_guard<std::mutex> lk(m->lock);
  DeviceGuard g(m->device);
  return m->timer.enable(enable != 0);
}

extern "C" int tbtkkpm_matrix_profile(tbtkkpm_matrix *m, double *recursion_ms, double *energy_ms,
                                      uint64_t *recursion_launches) {
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_profile: NULL handle");
  std::lock_guard<std::mutex> lk(m->lock);
  if (recursion_ms) *recursion_ms = m->timer.recursion_ms;
  if (energy_ms) *energy_ms = m->timer.energy_ms;
  if (recursion_launches) *recursion_launches = m->timer.step_launches;
  m->timer.recursion_ms = m->timer.energy_ms = 0;
  m->timer.step_launches = 0;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_device_count(int *count) {
  if (!count) return fail(TBTKKPM_ERR_ARGUMENT, "tbtkkpm_device_count: count is NULL");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_set_device(int device) {
  int n = 0;
  tbtkkpm_device_count(&n);
  if (device < 0 || device >= n)
    return fail(TBTKKPM_ERR_ARGUMENT, "tbtkkpm_set_device: device %d of %d", device, n);
  g_device = device;
  return TBTKKPM_OK;
}

// ---------------------------------------------------------------- C ABI: matrix

static int matrix_alloc(uint32_t N, uint64_t nnz, double scale, tbtkkpm_matrix **out) {
  int ndev = 0;
  tbtkkpm_device_count(&ndev);
  if (ndev == 0) return fail(TBTKKPM_ERR_CUDA, "no CUDA device available");
  auto *m = new tbtkkpm_matrix();
  m->device = current_device();
  m->N = N;
  m->nnz = nnz;
  m->scale = scale;
  DeviceGuard g(m->device);
  cudaError_t e = cudaStreamCreateWithFlags(&m->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete m;
    return cuda_fail(e, "cudaStreamCreate");
  }
  m->stream = m->own_stream;
  int rc;
  if ((rc = m->rowptr.reserve(sizeof(uint32_t) * ((size_t)N + 1))) ||
      (rc = m->col.reserve(sizeof(uint32_t) * std::max<uint64_t>(nnz, 1))) ||
      (rc = m->val2.reserve(sizeof(double2) * std::max<uint64_t>(nnz, 1)))) {
    tbtkkpm_matrix_destroy(m);
    return rc;
  }
  *out = m;
  return TBTKKPM_OK;
}

namespace {

// The smallest i in [0, n) for which bad(i) holds, else n.  The host checks
// of a large matrix run in chunks on up to 16 threads (one per 2^20 items).
template <typename F>
uint64_t first_bad(uint64_t n, F bad) {
  const uint64_t hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned T = (unsigned)std::min<uint64_t>(std::min<uint64_t>(16, hw), std::max<uint64_t>(1, n >> 20));
  if (T <= 1) {
    for (uint64_t i = 0; i < n; i++)
      if (bad(i)) return i;
    return n;
  }
  std::vector<uint64_t> first(T, n);
  std::vector<std::thread> th;
  const uint64_t chunk = (n + T - 1) / T;
  for (unsigned t = 0; t < T; t++)
    th.emplace_back([&, t] {
      const uint64_t a = t * chunk, b = std::min(n, a + chunk);
      for (uint64_t i = a; i < b; i++)
        if (bad(i)) {
          first[t] = i;
          return;
        }
    });
  for (auto &x : th) x.join();
  for (unsigned t = 0; t < T; t++)
    if (first[t] < n) return first[t];
  return n;
}

}  // namespace

extern "C" int tbtkkpm_matrix_create_csr(const uint32_t *rowptr, const uint32_t *col,
                                         const double *val, uint32_t N, double scale,
                                         tbtkkpm_matrix **out) {
  if (!out) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_create_csr: out is NULL");
  *out = nullptr;
  if (!rowptr || N == 0) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_create_csr: empty matrix");
  if (!(scale > 0))
    return fail(TBTKKPM_ERR_ARGUMENT,
                "matrix_create_csr: the scaleFactor=%g has to be larger than 0", scale);
  if (rowptr[0] != 0) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_create_csr: rowptr[0] != 0");
  const uint64_t dec = first_bad(N, [&](uint64_t r) { return rowptr[r + 1] < rowptr[r]; });
  if (dec < N)
    return fail(TBTKKPM_ERR_ARGUMENT, "matrix_create_csr: rowptr decreases at row %u", (uint32_t)dec);
  const uint64_t nnz = rowptr[N];
  if (nnz && (!col || !val)) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_create_csr: NULL arrays");
  // the first row with a column outside the basis, columns out of order or
  // a value that is not finite, then its message
  auto entry_bad = [&](uint32_t r, uint32_t k) -> int {
    if (col[k] >= N) return 1;
    if (k > rowptr[r] && col[k] <= col[k - 1]) return 2;
    if (!std::isfinite(val[2 * (uint64_t)k]) || !std::isfinite(val[2 * (uint64_t)k + 1])) return 3;
    return 0;
  };
  const uint64_t badrow = first_bad(N, [&](uint64_t r) {
    for (uint32_t k = rowptr[r]; k < rowptr[r + 1]; k++)
      if (entry_bad((uint32_t)r, k)) return true;
    return false;
  });
  if (badrow < N) {
    const uint32_t r = (uint32_t)badrow;
    for (uint32_t k = rowptr[r]; k < rowptr[r + 1]; k++) {
      const int why = entry_bad(r, k);
      if (why == 1)
        return fail(TBTKKPM_ERR_ARGUMENT, "matrix_create_csr: column %u of row %u >= N=%u",
                    col[k], r, N);
      if (why == 2)
        return fail(TBTKKPM_ERR_ARGUMENT,
                    "matrix_create_csr: columns of row %u not strictly ascending", r);
      if (why == 3)
        return fail(TBTKKPM_ERR_ARGUMENT,
                    "matrix_create_csr: value of row %u, column %u is not finite", r, col[k]);
    }
  }
  tbtkkpm_matrix *m = nullptr;
  int rc = matrix_alloc(N, nnz, scale, &m);
  if (rc) return rc;
  DeviceGuard g(m->device);
  cudaError_t e;
  if ((e = cudaMemcpyAsync(m->rowptr.ptr, rowptr, sizeof(uint32_t) * ((size_t)N + 1),
                           cudaMemcpyHostToDevice, m->stream)) != cudaSuccess ||
      (nnz && (e = cudaMemcpyAsync(m->col.ptr, col, sizeof(uint32_t) * nnz,
                                   cudaMemcpyHostToDevice, m->stream)) != cudaSuccess) ||
      (nnz && (e = cudaMemcpyAsync(m->val2.ptr, val, sizeof(double2) * nnz,
                                   cudaMemcpyHostToDevice, m->stream)) != cudaSuccess)) {
    tbtkkpm_matrix_destroy(m);
    return cuda_fail(e, "matrix_create_csr: upload");
  }
  if (nnz)
  {
    k_scale_values<<<blocks_for(nnz), 256, 0, m->stream>>>(nnz, 1 / scale,
                                                          (double2 *)m->val2.ptr);
    count_launches(1);
  }
  if ((rc = build_sell(m, m->stream))) {
    tbtkkpm_matrix_destroy(m);
    return rc;
  }
  if ((e = cudaStreamSynchronize(m->stream)) != cudaSuccess) {
    tbtkkpm_matrix_destroy(m);
    return cuda_fail(e, "matrix_create_csr: scale");
  }
  *out = m;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_create_triplets(const uint32_t *rows, const uint32_t *cols,
                                              const double *vals, uint64_t n, uint32_t N,
                                              double scale, tbtkkpm_matrix **out) {
  if (!out) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_create_triplets: out is NULL");
  *out = nullptr;
  if (N == 0) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_create_triplets: N is 0");
  if (!(scale > 0))
    return fail(TBTKKPM_ERR_ARGUMENT,
                "matrix_create_triplets: the scaleFactor=%g has to be larger than 0", scale);
  if (n && (!rows || !cols || !vals))
    return fail(TBTKKPM_ERR_ARGUMENT, "matrix_create_triplets: NULL arrays");
  const uint64_t i = first_bad(n, [&](uint64_t k) {
    return rows[k] >= N || cols[k] >= N || !std::isfinite(vals[2 * k]) ||
           !std::isfinite(vals[2 * k + 1]);
  });
  if (i < n) {
    if (rows[i] >= N || cols[i] >= N)
      return fail(TBTKKPM_ERR_ARGUMENT,
                  "matrix_create_triplets: entry %llu (%u, %u) outside the %u x %u basis",
                  (unsigned long long)i, rows[i], cols[i], N, N);
    return fail(TBTKKPM_ERR_ARGUMENT, "matrix_create_triplets: value of entry %llu is not finite",
                (unsigned long long)i);
  }
  int ndev = 0;
  tbtkkpm_device_count(&ndev);
  if (ndev == 0) return fail(TBTKKPM_ERR_CUDA, "no CUDA device available");
  const int dev = current_device();
  DeviceGuard g(dev);
  cudaStream_t st;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
  DevBuf d_rows, d_cols, d_vals, keys[2], order[2], head, pos, d_col, d_val, d_rowof, tmp;
  int rc = TBTKKPM_OK;
  uint64_t nnz = 0;
  const uint64_t nn = std::max<uint64_t>(n, 1);
  auto cleanup = [&]() {
    for (DevBuf *b : {&d_rows, &d_cols, &d_vals, &keys[0], &keys[1], &order[0], &order[1],
                      &head, &pos, &d_col, &d_val, &d_rowof, &tmp})
      b->release();
    cudaStreamDestroy(st);
  };
  if ((rc = d_rows.reserve(4 * nn)) || (rc = d_cols.reserve(4 * nn)) ||
      (rc = d_vals.reserve(16 * nn)) || (rc = keys[0].reserve(8 * nn)) ||
      (rc = keys[1].reserve(8 * nn)) || (rc = order[0].reserve(8 * nn)) ||
      (rc = order[1].reserve(8 * nn)) || (rc = head.reserve(4 * nn)) ||
      (rc = pos.reserve(4 * nn)) || (rc = d_col.reserve(4 * nn)) ||
      (rc = d_val.reserve(16 * nn)) || (rc = d_rowof.reserve(4 * nn))) {
    cleanup();
    return rc;
  }
  if (n) {
    cudaMemcpyAsync(d_rows.ptr, rows, 4 * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_cols.ptr, cols, 4 * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_vals.ptr, vals, 16 * n, cudaMemcpyHostToDevice, st);
    k_make_keys<<<blocks_for(n), 256, 0, st>>>(n, (uint32_t *)d_rows.ptr,
                                               (uint32_t *)d_cols.ptr, (uint64_t *)keys[0].ptr,
                                               (uint64_t *)order[0].ptr);
    cub::DoubleBuffer<uint64_t> kb((uint64_t *)keys[0].ptr, (uint64_t *)keys[1].ptr);
    cub::DoubleBuffer<uint64_t> vb((uint64_t *)order[0].ptr, (uint64_t *)order[1].ptr);
    size_t tbytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tbytes, kb, vb, (int64_t)n, 0, 64, st);
    size_t sbytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, sbytes, (uint32_t *)head.ptr, (uint32_t *)pos.ptr,
                                  (int64_t)n, st);
    if ((rc = tmp.reserve(std::max(tbytes, sbytes)))) {
      cleanup();
      return rc;
    }
    cub::DeviceRadixSort::SortPairs(tmp.ptr, tbytes, kb, vb, (int64_t)n, 0, 64, st);
    const uint64_t *sk = kb.Current();
    const uint64_t *so = vb.Current();
    k_mark_heads<<<blocks_for(n), 256, 0, st>>>(n, sk, (uint32_t *)head.ptr);
    count_launches(3);
    cub::DeviceScan::ExclusiveSum(tmp.ptr, sbytes, (uint32_t *)head.ptr, (uint32_t *)pos.ptr,
                                  (int64_t)n, st);
    k_fold_runs<<<blocks_for(n), 256, 0, st>>>(n, sk, so, (const double2 *)d_vals.ptr,
                                               (uint32_t *)head.ptr, (uint32_t *)pos.ptr,
                                               (uint32_t *)d_col.ptr, (double2 *)d_val.ptr,
                                               (uint32_t *)d_rowof.ptr);
    uint32_t last_pos = 0, last_head = 0;
    cudaMemcpyAsync(&last_pos, (uint32_t *)pos.ptr + (n - 1), 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last_head, (uint32_t *)head.ptr + (n - 1), 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) {
      cleanup();
      return cuda_fail(e, "matrix_create_triplets: sort");
    }
    nnz = (uint64_t)last_pos + last_head;
  }
  tbtkkpm_matrix *m = nullptr;
  if ((rc = matrix_alloc(N, nnz, scale, &m))) {
    cleanup();
    return rc;
  }
  if (nnz) {
    cudaMemcpyAsync(m->col.ptr, d_col.ptr, 4 * nnz, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(m->val2.ptr, d_val.ptr, 16 * nnz, cudaMemcpyDeviceToDevice, st);
    k_scale_values<<<blocks_for(nnz), 256, 0, st>>>(nnz, 1 / scale, (double2 *)m->val2.ptr);
  }
  k_rowptr<<<blocks_for(nnz + 1), 256, 0, st>>>(nnz, N, (uint32_t *)d_rowof.ptr,
                                                (uint32_t *)m->rowptr.ptr);
  count_launches(nnz ? 2 : 1);
  e = cudaStreamSynchronize(st);
  cleanup();
  if (e != cudaSuccess) {
    tbtkkpm_matrix_destroy(m);
    return cuda_fail(e, "matrix_create_triplets: build");
  }
  if ((rc = build_sell(m, m->stream))) {
    tbtkkpm_matrix_destroy(m);
    return rc;
  }
  *out = m;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_destroy(tbtkkpm_matrix *m) {
  if (!m) return TBTKKPM_OK;
  {
    DeviceGuard g(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    m->release_all();
    if (m->own_stream) cudaStreamDestroy(m->own_stream);
  }
  delete m;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_set_stream(tbtkkpm_matrix *m, void *cuda_stream) {
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_set_stream: NULL handle");
  std::lock_guard<std::mutex> lk(m->lock);
  DeviceGuard g(m->device);
  cudaStream_t next = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : m->own_stream;
  cudaError_t e = cudaStreamSynchronize(m->stream);
  if (e != cudaSuccess) return cuda_fail(e, "matrix_set_stream");
  m->stream = next;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_shape(const tbtkkpm_matrix *m, uint32_t *N, uint64_t *nnz) {
  if (!m) return fail(TBTKKPM_ERR_ARGUMENT, "matrix_shape: NULL handle");
  if (N) *N = m->N;
  if (nnz) *nnz = m->nnz;
  return TBTKKPM_OK;
}

extern "C" int tbtkkpm_matrix_download_csr(const tbtkkpm_matrix *m, uint32_t *rowptr,
                                           uint32_t *col, double *val) {
  if (!m || !rowptr || (m->nnz && (!col || !val)))
    return fail(TBTKKPM_ERR_ARGUMENT, "matrix_download_csr: NULL argument");
  DeviceGuard g(m->device);
  cudaError_t e;
  if ((e = cudaMemcpyAsync(rowptr, m->rowptr.ptr, 4 * ((size_t)m->N + 1),
                           cudaMemcpyDeviceToHost, m->stream)) != cudaSuccess)
    return cuda_fail(e, "matrix_download_csr");
  if (m->nnz) {
    cudaMemcpyAsync(col, m->col.ptr, 4 * m->nnz, cudaMemcpyDeviceToHost, m->stream);
    cudaMemcpyAsync(val, m->val2.ptr, 16 * m->nnz, cudaMemcpyDeviceToHost, m->stream);
  }
  if ((e = cudaStreamSynchronize(m->stream)) != cudaSuccess)
    return cuda_fail(e, "matrix_download_csr");
  return TBTKKPM_OK;
}
