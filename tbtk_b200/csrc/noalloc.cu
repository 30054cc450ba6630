// tbtkkpm_moments_noalloc: Chebyshev moments without any device allocation.
//
// Some callers cannot call cudaMalloc: code running inside another
// framework's memory pool, code that must not grow the device footprint
// after start-up, or code that holds the device memory budget for itself.
// This entry point takes the matrix and the output in the caller's device
// buffers and keeps its only scratch, the two recursion vectors and the
// damping factors, in a fixed array compiled into the library.
//
// The array is kNoAllocScratchBytes (32 MiB) of device memory.  A GPU holds
// it from the moment this code is loaded onto that device (with CUDA's lazy
// module loading: the first call there) until the process exits.  Host code
// must not pass the array's name to a kernel (on the host that name is a
// stand-in, not a device address); the first call on a device, with that
// device current, looks the address up with cudaGetSymbolAddress and caches
// it for the process.  A cudaDeviceReset invalidates that address (and every
// other handle of this library on the device): do not call this entry point
// on a device after resetting it.  All calls share the array and it keeps
// the previous call's contents: each call clears the vectors it uses, and
// calls that overlap on the GPU race (serialise them on one stream).  Every
// call is synchronous (it copies host data and waits for its stream), so no
// call can be captured into a CUDA graph.
#include "tbtkkpm.h"
#include "kpm_host.h"
#include "kpm_kernels.cuh"

#include <cmath>
#include <mutex>
#include <vector>

namespace tbtkkpm {

namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;

// The scratch: [2][N] complex128 vectors, then [M] damping numerators, then
// one status word.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_lock;
void *g_scratch_addr[64] = {nullptr};

// Device address of the scratch on the current device (looked up once).
int scratch_address(int device, unsigned char **out) {
  std::lock_guard<std::mutex> lk(g_scratch_lock);
  if (device < 0 || device >= 64) return fail(TBTKKPM_ERR_ARGUMENT, "moments_noalloc: device %d", device);
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "moments_noalloc: cudaGetSymbolAddress");
    g_scratch_addr[device] = p;
  }
  *out = static_cast<unsigned char *>(g_scratch_addr[device]);
  return TBTKKPM_OK;
}

// The caller's rowptr: rowptr[0] == 0, never decreasing, rowptr[N] == nnz;
// a violation sets status bit 4 (checked before any recursion step runs).
__global__ void noalloc_check_rowptr(uint32_t N, uint64_t nnz, const uint32_t *__restrict__ rowptr,
                                     unsigned *status) {
  const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= N) return;
  const uint32_t a = rowptr[row], b = rowptr[row + 1];
  if (a > b || b > nnz || (row == 0 && a != 0) || (row == N - 1 && b != nnz))
    atomicOr(status, 4u);
}

// One step on the caller's CSR, values scaled on the fly exactly as the
// matrix handles store them: v1 = v*(1/s) for the first step, 2*v1 after
// (ChebyshevExpander.cpp:147,168), each complex product in the reference's
// operation order.  Column indices out of range set status bit 1 and are
// skipped; entry ranges are clamped to [0, nnz) (rowptr is checked first).
__global__ void noalloc_step(uint32_t N, uint64_t nnz, const uint32_t *__restrict__ rowptr,
                             const uint32_t *__restrict__ col, const double2 *__restrict__ val,
                             double inv, bool first, const double2 *__restrict__ x,
                             double2 *__restrict__ y, unsigned *status) {
  const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= N) return;
  double2 acc = first ? make_double2(0.0, 0.0) : make_double2(-y[row].x, -y[row].y);
  const uint32_t k1 = (uint32_t)min((uint64_t)rowptr[row + 1], nnz);
  const uint32_t k0 = min(rowptr[row], k1);
  for (uint32_t k = k0; k < k1; k++) {
    const uint32_t c = col[k];
    if (c >= N) {
      atomicOr(status, 1u);
      continue;
    }
    double2 v = cmul_exact(val[k], make_double2(inv, 0.0));
    if (!first) v = cmul_exact(v, make_double2(2.0, 0.0));
    acc = cadd_exact(acc, cmul_exact(v, x[c]));
  }
  y[row] = acc;
}

// mu[k][n] = j_n[to_k]; to-indices out of range set status bit 2.
__global__ void noalloc_gather(uint32_t N, uint32_t K, uint32_t M, uint32_t n,
                               const uint32_t *__restrict__ to, const double2 *__restrict__ j,
                               double2 *mu, unsigned *status) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  const uint32_t t = to[k];
  if (t >= N) {
    atomicOr(status, 2u);
    mu[(uint64_t)k * M + n] = make_double2(0.0, 0.0);
    return;
  }
  mu[(uint64_t)k * M + n] = j[t];
}

__global__ void noalloc_seed(uint32_t from, double2 *x) { x[from] = make_double2(1.0, 0.0); }

// mu[k][n] = mu[k][n]*a[n]/b (ChebyshevExpander.cpp:190-196).
__global__ void noalloc_damp(uint32_t K, uint32_t M, const double *a, double b, double2 *mu) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint64_t)K * M) return;
  const double an = a[i % M];
  const double2 c = mu[i];
  mu[i] = make_double2(__ddiv_rn(__dmul_rn(c.x, an), b), __ddiv_rn(__dmul_rn(c.y, an), b));
}

inline unsigned blocks(uint64_t n, unsigned bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

}  // namespace tbtkkpm

using namespace tbtkkpm;

extern "C" int tbtkkpm_moments_noalloc(const uint32_t *d_rowptr, const uint32_t *d_col,
                                       const double *d_val, uint32_t N, uint64_t nnz,
                                       double scale, uint32_t from, const uint32_t *d_to,
                                       uint32_t K, uint32_t M, double broadening,
                                       double *d_mu_out, void *stream) {
  if (!d_rowptr || N == 0) return fail(TBTKKPM_ERR_ARGUMENT, "moments_noalloc: empty matrix");
  if (nnz > 0xffffffffull)
    return fail(TBTKKPM_ERR_ARGUMENT, "moments_noalloc: nnz=%llu past 32-bit entry indices",
                (unsigned long long)nnz);
  if (!(scale > 0))
    return fail(TBTKKPM_ERR_ARGUMENT,
                "moments_noalloc: the scaleFactor=%g has to be larger than 0", scale);
  if (M == 0) return fail(TBTKKPM_ERR_ARGUMENT, "moments_noalloc: numCoefficients has to be larger than 0");
  if (from >= N)
    return fail(TBTKKPM_ERR_ARGUMENT, "moments_noalloc: from index %u outside the basis of size %u",
                from, N);
  if (K == 0) return TBTKKPM_OK;
  if (!d_to || !d_mu_out || (nnz && (!d_col || !d_val)))
    return fail(TBTKKPM_ERR_ARGUMENT, "moments_noalloc: NULL device buffer");
  if (!std::isfinite(broadening)) return fail(TBTKKPM_ERR_ARGUMENT, "moments_noalloc: broadening not finite");
  const size_t vec_bytes = sizeof(double2) * (size_t)N;
  const size_t need = 2 * vec_bytes + sizeof(double) * (size_t)M + 256;
  if (need > kNoAllocScratchBytes)
    return fail(TBTKKPM_ERR_ARGUMENT,
                "moments_noalloc: N=%u and M=%u need %zu bytes of scratch, more than its fixed "
                "%zu bytes (32*N + 8*M + 256 <= 32 MiB); use tbtkkpm_moments",
                N, M, need, kNoAllocScratchBytes);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "moments_noalloc: cudaGetDevice");
  unsigned char *base = nullptr;
  int rc = scratch_address(dev, &base);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double2 *v0 = reinterpret_cast<double2 *>(base);
  double2 *v1 = reinterpret_cast<double2 *>(base + vec_bytes);
  double *damp = reinterpret_cast<double *>(base + 2 * vec_bytes);
  unsigned *status =
      reinterpret_cast<unsigned *>(base + ((2 * vec_bytes + sizeof(double) * M + 15) / 16) * 16);
  double2 *mu = reinterpret_cast<double2 *>(d_mu_out);
  const double2 *val = reinterpret_cast<const double2 *>(d_val);
  if ((e = cudaMemsetAsync(base, 0, 2 * vec_bytes, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(status, 0, sizeof(unsigned), st)) != cudaSuccess)
    return cuda_fail(e, "moments_noalloc: clear");
  // the caller's rowptr is checked before a step reads entries through it
  noalloc_check_rowptr<<<blocks(N, 256), 256, 0, st>>>(N, nnz, d_rowptr, status);
  unsigned flag = 0;
  if ((e = cudaMemcpyAsync(&flag, status, sizeof(unsigned), cudaMemcpyDeviceToHost, st)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_fail(e, "moments_noalloc: rowptr check");
  if (flag & 4u)
    return fail(TBTKKPM_ERR_ARGUMENT,
                "moments_noalloc: rowptr is not a CSR row pointer of nnz=%llu entries "
                "(rowptr[0] == 0, non-decreasing, rowptr[N] == nnz)",
                (unsigned long long)nnz);
  noalloc_seed<<<1, 1, 0, st>>>(from, v0);
  noalloc_gather<<<blocks(K, 128), 128, 0, st>>>(N, K, M, 0, d_to, v0, mu, status);
  const double inv = 1 / scale;
  double2 *cur = v0, *prev = v1;
  for (uint32_t n = 1; n < M; n++) {
    noalloc_step<<<blocks(N, 256), 256, 0, st>>>(N, nnz, d_rowptr, d_col, val, inv, n == 1, cur,
                                                prev, status);
    noalloc_gather<<<blocks(K, 128), 128, 0, st>>>(N, K, M, n, d_to, prev, mu, status);
    std::swap(cur, prev);
  }
  count_launches(3 + 2 * (uint64_t)(M - 1));
  double b = 1;
  if (broadening != 0) {
    // the host's libm, exactly as ChebyshevExpander.cpp:192-195
    std::vector<double> a(M);
    const double lambda = broadening * M;
    for (uint32_t n = 0; n < M; n++) a[n] = std::sinh(lambda * (1 - n / (double)M));
    b = std::sinh(lambda);
    if ((e = cudaMemcpyAsync(damp, a.data(), sizeof(double) * M, cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
      return cuda_fail(e, "moments_noalloc: damping factors");
    noalloc_damp<<<blocks((uint64_t)K * M, 256), 256, 0, st>>>(K, M, damp, b, mu);
    count_launches(1);
  }
  if ((e = cudaMemcpyAsync(&flag, status, sizeof(unsigned), cudaMemcpyDeviceToHost, st)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_fail(e, "moments_noalloc: run");
  if (flag & 1u) return fail(TBTKKPM_ERR_ARGUMENT, "moments_noalloc: a column index is >= N");
  if (flag & 2u) return fail(TBTKKPM_ERR_ARGUMENT, "moments_noalloc: a to index is >= N");
  return TBTKKPM_OK;
}
