/* tbtkkpm — the kernel-polynomial (Chebyshev) path of TBTK on NVIDIA B200.
 *
 * A C ABI over hand-written sm_100a kernels.  It replaces the device side
 * of TBTK's Solver::ChebyshevExpander (Lib/src/cuda/ChebyshevSolver.cu) and
 * the per-site loop of PropertyExtractor::ChebyshevExpander::calculateLDOS.
 * Plain pointers and sizes only; complex numbers are interleaved
 * (re, im) doubles; every index is a TBTK basis number (the caller maps
 * Index -> basis with HoppingAmplitudeSet::getBasisIndex).
 *
 * Errors: every entry point returns TBTKKPM_OK (0) or a negative status and
 * never exits the process; tbtkkpm_last_error() gives the message of the
 * calling thread's last failure.  (The reference reports errors through
 * TBTKAssert/TBTKExit, Lib/include/Utilities/TBTK/TBTKMacros.h:55-94, which
 * print and exit(1); a TBTK-side caller turns a non-zero status back into
 * TBTKExit.)
 *
 * Threads: calls on distinct handles may run concurrently; each handle owns
 * one CUDA stream on the device that was current when it was created.  Calls
 * that return host results synchronise that stream before returning.
 */
#ifndef TBTKKPM_H
#define TBTKKPM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TBTKKPM_API __attribute__((visibility("default")))
#else
#define TBTKKPM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status */

#define TBTKKPM_OK 0
#define TBTKKPM_ERR_ARGUMENT -1   /* an argument is out of range */
#define TBTKKPM_ERR_CUDA -2       /* a CUDA call failed */
#define TBTKKPM_ERR_MEMORY -3     /* device memory or HBM budget exhausted */
#define TBTKKPM_ERR_TIMEOUT -4    /* a bounded device wait ran out */
#define TBTKKPM_ERR_UNSUPPORTED -5/* combination not available */
#define TBTKKPM_ERR_STATE -6      /* handle in the wrong state */
#define TBTKKPM_ERR_CANCELLED -7  /* a server request was cancelled */

/* Message of the calling thread's last failed call ("" if none). */
TBTKKPM_API const char *tbtkkpm_last_error(void);

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
TBTKKPM_API int tbtkkpm_version(void);

/* Number of CUDA devices (the reference's GPUResourceManager device table,
 * Lib/src/cuda/GPUResourceManager.cu:28-39). */
TBTKKPM_API int tbtkkpm_device_count(int *count);

/* Selects the device later handle creations on this thread use. */
TBTKKPM_API int tbtkkpm_set_device(int device);

/* Number of kernels this process has launched through the library.  (No
 * reference counterpart: instrumentation for benchmarks.) */
TBTKKPM_API uint64_t tbtkkpm_kernel_launches(void);

/* ------------------------------------------------------------ types */

/* Green's function type, the order of Solver::ChebyshevExpander::Type
 * (Lib/include/TBTK/Solver/ChebyshevExpander.h:203-208). */
#define TBTKKPM_ADVANCED 0
#define TBTKKPM_RETARDED 1
#define TBTKKPM_PRINCIPAL 2
#define TBTKKPM_NONPRINCIPAL 3

/* Recursion precision.
 * FP64: complex128 vectors, the reference's operation order (moments are
 *   bit-identical to calculateCoefficientsCPU).
 * MIXED: complex64 vectors in HBM, FP64 arithmetic in registers, FP64
 *   moments, damping and energy sums.  For LDOS (a source's only to-index is
 *   itself) the recursion runs to j_{M/2} only and takes two moments per
 *   step from FP64 dot products: mu_{2n} = 2<j_n|j_n> - mu_0,
 *   mu_{2n+1} = 2<j_{n+1}|j_n> - mu_1 (H Hermitian).
 * MIXED_DIRECT: MIXED with every moment gathered directly (no dot-product
 *   identities), M-1 steps. */
#define TBTKKPM_FP64 0
#define TBTKKPM_MIXED 1
#define TBTKKPM_MIXED_DIRECT 2

typedef struct tbtkkpm_matrix tbtkkpm_matrix;
typedef struct tbtkkpm_table tbtkkpm_table;

/* ------------------------------------------------------------ matrix */

/* Device copy of H/s from a CSR matrix in TBTK's layout: row = basis(to),
 * col = basis(from), columns ascending within a row, no duplicates
 * (HoppingAmplitudeSet::getSparseMatrix() after setStorageFormat(CSR),
 * Lib/include/Core/TBTK/HoppingAmplitudeSet.h:397-424).  rowptr has N+1
 * entries.  The values are scaled on the device exactly as
 * calculateCoefficientsCPU scales them (`*= 1/scaleFactor` then `*= 2`,
 * Lib/src/Solver/ChebyshevExpander.cpp:147,168) and stored in sliced ELL.
 * scale must be > 0 (ChebyshevExpander.h:394-403).  A NaN or infinite
 * value is rejected with TBTKKPM_ERR_ARGUMENT before any device work (the
 * reference accepts it and returns NaN moments). */
TBTKKPM_API int tbtkkpm_matrix_create_csr(
	const uint32_t *rowptr, const uint32_t *col, const double *val,
	uint32_t N, double scale, tbtkkpm_matrix **out);

/* Same from unsorted (row, col, value) triplets in HoppingAmplitudeSet
 * iteration order; sorting and duplicate summation run on the device with
 * the semantics of SparseMatrix::constructCSX (SparseMatrix.h:1375-1551;
 * duplicates d0, d1, d2 of one entry sum as d0 + (d1 + d2)). */
TBTKKPM_API int tbtkkpm_matrix_create_triplets(
	const uint32_t *rows, const uint32_t *cols, const double *vals,
	uint64_t n, uint32_t N, double scale, tbtkkpm_matrix **out);

TBTKKPM_API int tbtkkpm_matrix_destroy(tbtkkpm_matrix *m);

/* Runs this handle's work on the caller's CUDA stream (a cudaStream_t of
 * the handle's device) instead of its own; NULL restores its own stream.
 * (No reference counterpart: the reference uses the default stream.) */
TBTKKPM_API int tbtkkpm_matrix_set_stream(tbtkkpm_matrix *m, void *cuda_stream);

/* Basis size and stored nonzeros of a matrix. */
TBTKKPM_API int tbtkkpm_matrix_shape(const tbtkkpm_matrix *m, uint32_t *N, uint64_t *nnz);

/* Downloads the scaled CSR (values 2/s * H, i.e. what the recursion
 * multiplies by after step 1) for checking; rowptr N+1, col/val nnz. */
TBTKKPM_API int tbtkkpm_matrix_download_csr(
	const tbtkkpm_matrix *m, uint32_t *rowptr, uint32_t *col, double *val);

/* Phase timing of the calls on this handle, with CUDA events recorded on
 * the handle's stream around the recursion and around the energy sums.
 * tbtkkpm_matrix_profile returns the milliseconds and recursion-step
 * launches accumulated since the previous read and resets them.  (No
 * reference counterpart: the reference's Timer::tick/tock,
 * Lib/include/Utilities/TBTK/Timer.h:75-105, is host wall time.) */
TBTKKPM_API int tbtkkpm_matrix_set_profiling(tbtkkpm_matrix *m, int enable);
TBTKKPM_API int tbtkkpm_matrix_profile(
	tbtkkpm_matrix *m, double *recursion_ms, double *energy_ms,
	uint64_t *recursion_launches);

/* ------------------------------------------------------------ moments */

/* Chebyshev moments mu[k][n] = <to_k| T_n(H/s) |from>, n = 0..M-1, for K
 * to-indices, then Lorentz damping sinh(lambda(1-n/M))/sinh(lambda),
 * lambda = broadening*M (none if broadening == 0).  mu_out is [K][M]
 * complex.  Replaces Solver::ChebyshevExpander::calculateCoefficientsGPU
 * (Lib/src/cuda/ChebyshevSolver.cu:74-648) and matches
 * calculateCoefficientsCPU (Lib/src/Solver/ChebyshevExpander.cpp:103-199)
 * bit for bit at TBTKKPM_FP64. */
TBTKKPM_API int tbtkkpm_moments(
	tbtkkpm_matrix *m, uint32_t from, const uint32_t *to, uint32_t K,
	uint32_t M, double broadening, double *mu_out);

/* tbtkkpm_moments for callers that cannot allocate device memory (code
 * inside another framework's memory pool, or under a fixed device-memory
 * budget).  It allocates nothing: the matrix (CSR as for
 * tbtkkpm_matrix_create_csr, unscaled: d_rowptr N+1 entries, d_col and
 * d_val nnz entries) and the output are the caller's device buffers (d_to:
 * K basis indices; d_mu_out: [K][M] complex, damped as tbtkkpm_moments), and
 * its scratch is a fixed 32 MiB array compiled into the library, which a GPU
 * holds from the first call there (when the library's device code loads)
 * until the process exits.  Sizes with 32*N + 8*M + 256 > 32 MiB are
 * rejected (use tbtkkpm_moments).  The first call on a device looks the
 * array up on the current device and caches the address for the process; a
 * cudaDeviceReset of that device invalidates it, so do not call this after
 * resetting the device.  Calls share the array: each call clears what it
 * uses, and calls that overlap on the GPU race.  Work runs on `stream`
 * (NULL: the default stream); every call is synchronous (it copies host
 * data and waits for the stream), so it cannot be captured into a CUDA
 * graph.  The device checks d_rowptr first (rowptr[0] == 0, non-decreasing,
 * rowptr[N] == nnz), then skips column and to indices >= N; any of these
 * returns TBTKKPM_ERR_ARGUMENT.  (No counterpart in the reference.) */
TBTKKPM_API int tbtkkpm_moments_noalloc(
	const uint32_t *d_rowptr, const uint32_t *d_col, const double *d_val,
	uint32_t N, uint64_t nnz, double scale, uint32_t from,
	const uint32_t *d_to, uint32_t K, uint32_t M, double broadening,
	double *d_mu_out, void *stream);

/* Batched moments: B source vectors (from[b]) advance together as one
 * SpMM-style recursion.  to[k] belongs to source to_owner[k]; mu_out is
 * [K][M] complex in the order of to[].  precision is TBTKKPM_FP64 or
 * TBTKKPM_MIXED.  err_out (may be NULL) receives, per to-index, an
 * estimate of max_n |mu_n - mu_n(FP64)| / max_n |mu_n| (0 at FP64). */
TBTKKPM_API int tbtkkpm_moments_batched(
	tbtkkpm_matrix *m, const uint32_t *from, uint32_t B,
	const uint32_t *to, const uint32_t *to_owner, uint32_t K, uint32_t M,
	double broadening, int precision, double *mu_out, double *err_out);

/* ------------------------------------------------------------ energy grid */

/* Lookup table T[n][e] = (1/s)(-2i/sqrt(1-x^2)) exp(-i n acos x)/(1+delta_n0),
 * x = energies[e]/s, generated on the device (generateLookupTable,
 * Lib/src/Solver/ChebyshevExpander.cpp:201-270).  The energies must lie in
 * (-s, s) (ChebyshevExpander.cpp:221-236). */
TBTKKPM_API int tbtkkpm_table_create(
	uint32_t M, const double *energies, uint32_t E, double scale,
	tbtkkpm_table **out);

/* Same from a table computed on the host ([M][E] complex), the layout
 * loadLookupTableGPU uploads (Lib/src/cuda/ChebyshevSolver.cu:672-760). */
TBTKKPM_API int tbtkkpm_table_upload(
	uint32_t M, uint32_t E, const double *table, tbtkkpm_table **out);

/* A table handle without the M x E table: the energy sums of every call
 * that takes it (tbtkkpm_greens, tbtkkpm_ldos, tbtkkpm_ldos_sites, the
 * properties) run Clenshaw recurrences over T_n(E/s) and U_n(E/s) per
 * energy instead (O(M) arithmetic per vector and energy, 8 E bytes of
 * device memory instead of 16 M E).  Results equal the table sums up to
 * rounding (~1e-13 relative).  Same arguments and checks as
 * tbtkkpm_table_create.  (A table-free energy-sum variant; no
 * reference counterpart: generateGreensFunctionCPU without a table,
 * ChebyshevExpander.cpp:363-433, evaluates e^{-in acos x} per term.) */
TBTKKPM_API int tbtkkpm_table_create_clenshaw(
	uint32_t M, const double *energies, uint32_t E, double scale,
	tbtkkpm_table **out);

/* A table handle on the grid of Chebyshev nodes: E energies (E a power of
 * two, 1 <= E <= 4096) E_e = -s cos(pi (2e + 1) / (2E)), ascending, are
 * written to energies_out[E].  The energy sums of every call that takes
 * the handle run one FFT of length 2E per coefficient vector (O(E log E)
 * arithmetic per vector instead of the table's O(M E) multiply-adds and
 * 16 M E table bytes; 32 E bytes of device memory).  M is the most
 * coefficients a call may pass; any M works (terms beyond 2E fold onto the
 * transform).  Results are the sums at the exact node angles (~1e-13
 * relative); the lookup-table sums on the same energies agree to ~1e-11
 * away from the band edges, less at the outermost nodes, where the
 * table's acos of the stored energy is ill-conditioned (a phase error of
 * about n eps / sqrt(1 - x^2)).  The grid is not uniform: the properties
 * that integrate over energy with a spacing dE (density, magnetization,
 * expectation values) assume a uniform grid and are not meant for it.
 * (The discrete-cosine-transform energy-sum variant; no reference
 * counterpart: the reference sums over a uniform Range,
 * Lib/src/Solver/ChebyshevExpander.cpp:201-270,277-435.) */
TBTKKPM_API int tbtkkpm_table_create_chebyshev(
	uint32_t M, uint32_t E, double scale, double *energies_out,
	tbtkkpm_table **out);

TBTKKPM_API int tbtkkpm_table_destroy(tbtkkpm_table *t);

/* Green's functions G[k][e] of one type from K damped coefficient vectors
 * mu[k][n] (n < M of the table), summed in the reference's order
 * (generateGreensFunctionCPU with a table, ChebyshevExpander.cpp:324-361;
 * the reference GPU path only had the Retarded type,
 * ChebyshevSolver.cu:650-670,811-818).  G_out is [K][E] complex. */
TBTKKPM_API int tbtkkpm_greens(
	tbtkkpm_table *t, const double *mu, uint32_t K, int type, double *G_out);

/* LDOS[k][e] = Im(G_NonPrincipal[k][e]) / pi (calculateLDOSCallback,
 * Lib/src/PropertyExtractor/ChebyshevExpander.cpp:661-684).  [K][E]. */
TBTKKPM_API int tbtkkpm_ldos(
	tbtkkpm_table *t, const double *mu, uint32_t K, double *ldos_out);

/* Autotuner.  Times every compiled recursion-step configuration (threads
 * per row, complex values per thread, register cap) that serves batches of
 * B sources at this precision on this matrix, probe_steps steps each with
 * CUDA events on the handle's stream, and keeps the fastest for later calls
 * on this handle.  ldos != 0 tunes the kernels tbtkkpm_ldos_sites uses (the
 * dot-product variant at TBTKKPM_MIXED), 0 those of the moment calls.
 * Outputs (may be NULL): the chosen configuration and its ms per step.
 * tbtkkpm_matrix_set_config installs a known choice without timing.
 * (No reference counterpart.) */
TBTKKPM_API int tbtkkpm_matrix_autotune(
	tbtkkpm_matrix *m, uint32_t B, int precision, int ldos,
	uint32_t probe_steps, int *tpr, int *vpt, int *minb, double *ms_per_step);
TBTKKPM_API int tbtkkpm_matrix_set_config(
	tbtkkpm_matrix *m, uint32_t B, int precision, int ldos, int tpr, int vpt,
	int minb);

/* Lists the compiled step configurations of the kernels a call at this
 * precision uses as (tpr, vpt, variant) triples into out[3*cap]; returns
 * their number (-1 for an unknown precision).  variant 1..4 is the register
 * cap (min blocks per SM) of a register-staged kernel; 100 + 10*S + W is a
 * bulk-copy kernel with a ring of S stages per warp and W warps per block;
 * 10000 + 1000*S + 10*WMAX + W a cp.async-staged kernel.  Real-vector
 * kernels (real matrices at the mixed precisions): cap + 100*8 (802, 803)
 * keeps the doubling dot sums in shared memory instead of registers.
 * (No reference counterpart.) */
TBTKKPM_API int tbtkkpm_step_configs(int precision, int ldos, int *out, int cap);

/* Real Hamiltonians.  When every scaled value 2H/s of a matrix has a zero
 * imaginary part, the mixed precisions (TBTKKPM_MIXED, TBTKKPM_MIXED_DIRECT)
 * run on real float vectors instead of complex64 ones: every Chebyshev
 * vector of a real matrix started from basis vectors is real, and the real
 * kernels give the same moments (value, 0) with half the vector bytes.
 * The FP64 precision keeps complex128 vectors (the reference's data).
 * set_real(m, 0) turns the real vectors off (1, the default, allows them);
 * tbtkkpm_matrix_real reports whether the values are real and whether the
 * real vectors are in use; tbtkkpm_matrix_step_configs lists the step
 * configurations this matrix's calls choose from (as tbtkkpm_step_configs).
 * (No reference counterpart: the reference always uses complex<double>.) */
TBTKKPM_API int tbtkkpm_matrix_set_real(tbtkkpm_matrix *m, int enable);
TBTKKPM_API int tbtkkpm_matrix_real(tbtkkpm_matrix *m, int *values_real, int *in_use);
TBTKKPM_API int tbtkkpm_matrix_step_configs(
	tbtkkpm_matrix *m, int precision, int ldos, int *out, int cap);

/* FP64 head of TBTKKPM_MIXED doubling runs.  The doubled moments pick up
 * the FP32 rounding of the first steps, while the Chebyshev vectors still
 * sit on the few rows around their source; so a doubling run takes its
 * first `steps` steps (default 32, at most M/2 - 1) in FP64 on the rows
 * those steps reach, and the FP32 recursion starts from j_{q-1}, j_q.  This
 * needs a structurally symmetric pattern (checked when the matrix is made;
 * a Hermitian matrix has one) and a ball of at most 6144 rows (else the
 * batch stops its head at the last step that fits).  steps = 0 turns the
 * head off.  tbtkkpm_matrix_fp64_head reports the setting and whether the
 * pattern allows a head.  (No reference counterpart.) */
TBTKKPM_API int tbtkkpm_matrix_set_fp64_head(tbtkkpm_matrix *m, uint32_t steps);

/* Bound of each wait of the tile-staged recursion steps on this handle for
 * rows staged in shared memory (polls of the mbarrier; default
 * TBTKKPM_WAIT_DEFAULT).  A wait that runs out ends the step early, its
 * issued copies are waited for with the default bound, and the call returns
 * TBTKKPM_ERR_TIMEOUT; the handle stays usable.  polls = 0 makes every
 * such wait give up at once, which tests that path.  (No reference
 * counterpart: the reference's device waits are unbounded,
 * Lib/src/Utilities/GPUResourceManager.cpp:52-73.) */
#define TBTKKPM_WAIT_DEFAULT 0xffffffffu
TBTKKPM_API int tbtkkpm_matrix_set_wait_limit(tbtkkpm_matrix *m, uint32_t polls);
TBTKKPM_API int tbtkkpm_matrix_fp64_head(
	tbtkkpm_matrix *m, uint32_t *steps, int *pattern_symmetric);

/* Sources per recursion batch.  tbtkkpm_moments_batched and
 * tbtkkpm_ldos_sites split their sources into batches of at most this many
 * and run the batches one after another; each batch reads the matrix once
 * per step.  width 0 (the default) is the library's choice: 128 for
 * TBTKKPM_MIXED LDOS runs (the doubling step of 256 sources measured 20%
 * slower per source than two batches of 128, on real and complex
 * matrices), otherwise the maximum, 128 at TBTKKPM_FP64 and 256 at the
 * mixed precisions.  Widths above the maximum are rejected.
 * Results at TBTKKPM_FP64 and the directly gathered moments do not depend
 * on the width; doubled moments may differ in the last bits (their dot
 * products are summed in an order set by the batch's step configuration).
 * tbtkkpm_matrix_batch_width reports the width a call of this precision
 * uses (ldos != 0: tbtkkpm_ldos_sites, 0: the moment calls).
 * (No reference counterpart: the reference runs one source per recursion.) */
TBTKKPM_API int tbtkkpm_matrix_set_batch_width(
	tbtkkpm_matrix *m, int precision, uint32_t width);
TBTKKPM_API int tbtkkpm_matrix_batch_width(
	tbtkkpm_matrix *m, int precision, int ldos, uint32_t *width);

/* LDOS at B sites in one call: the moments <site|T_n|site> of all sites run
 * as one batched recursion, are damped and summed over the table's energy
 * grid on the device; only the [B][E] result crosses to the host.
 * Replaces the per-site loop of PropertyExtractor::ChebyshevExpander::
 * calculateLDOS (ChebyshevExpander.cpp:475-505 through
 * PropertyExtractor.h:849-894).  err_out (may be NULL) receives per site:
 * 0 at TBTKKPM_FP64; -1 at TBTKKPM_MIXED_DIRECT (no estimate); at
 * TBTKKPM_MIXED (doubling) 4 sqrt(2) times the largest gap between the
 * doubled and the directly gathered moments over 2 <= n <= M/2, relative to
 * max_n |mu_n| (measured against the FP64 path on 240 solves of a
 * 1000-model batch: 0.75x to 8x the LDOS's relative error). */
TBTKKPM_API int tbtkkpm_ldos_sites(
	tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *sites, uint32_t B,
	double broadening, int precision, double *ldos_out, double *err_out);

/* ------------------------------------------------------------ other properties
 *
 * PropertyExtractor::ChebyshevExpander's spin-polarized LDOS, density,
 * magnetization and expectation values
 * (Lib/src/PropertyExtractor/ChebyshevExpander.cpp:297-327,584-720).  The
 * reference computes one recursion per (to, from) pair; these run every
 * pair of a call as targets of one batched recursion
 * (tbtkkpm_moments_batched) and one NonPrincipal energy sum
 * (tbtkkpm_greens), then form the property with the reference's expression
 * and order.  Energies are the table's; occupation[e] is the equilibrium
 * occupation at energy e (the reference's
 * PropertyExtractor::getThermodynamicEquilibriumOccupation, from the
 * model's statistics, temperature and chemical potential) and dE the window
 * spacing (energyWindow[1] - energyWindow[0]).  A site with a spin subindex
 * is given by its spin-up and spin-down basis rows.  precision as for
 * tbtkkpm_moments_batched. */

/* out [S][E][2][2] complex: entry (a, b) = -i G_NP(to = spin a, from = spin
 * b)(E_e) / pi (calculateSP_LDOSCallback, :686-720). */
TBTKKPM_API int tbtkkpm_spin_polarized_ldos(
	tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *up,
	const uint32_t *down, uint32_t S, double broadening, int precision,
	double *out);

/* out[s] = sum_e occupation[e] Im G_NP(s, s)(E_e) / pi dE
 * (calculateDensityCallback, :584-616). */
TBTKKPM_API int tbtkkpm_density(
	tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *sites, uint32_t S,
	double broadening, int precision, const double *occupation, double dE,
	double *out);

/* out [S][2][2] complex = sum_e occupation[e] (-i) G_NP(a, b)(E_e) / pi dE
 * (calculateMAGCallback, :618-659). */
TBTKKPM_API int tbtkkpm_magnetization(
	tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *up,
	const uint32_t *down, uint32_t S, double broadening, int precision,
	const double *occupation, double dE, double *out);

/* out [P] complex = -sum_e occupation[e] conj(i G_NP(to_p, from_p)(E_e)) dE
 * / pi (calculateExpectationValue, :297-327). */
TBTKKPM_API int tbtkkpm_expectation_values(
	tbtkkpm_matrix *m, tbtkkpm_table *t, const uint32_t *to,
	const uint32_t *from, uint32_t P, double broadening, int precision,
	const double *occupation, double dE, double *out);

/* ------------------------------------------------------------ server
 *
 * A device-resident LDOS and Green's-function service over many models (no
 * reference counterpart: the reference answers one calculateLDOS or
 * calculateGreensFunction call at a time,
 * Lib/src/PropertyExtractor/ChebyshevExpander.cpp:96-295,475-505).  Each
 * model owns `width` lanes; a request (model, up to `width` sites or
 * (to, from) pairs, M moments, broadening) takes free lanes at the next
 * step boundary, one lane per source, and one kernel launch per step
 * advances every lane of every resident model (continuous batching).
 * Lanes run complex64 (or, for real models, float) vectors with FP64
 * arithmetic and FP64 moments; LDOS requests and Green's-function requests
 * whose pairs are all diagonal use the doubling identities, other
 * Green's-function requests gather every moment directly.  An output whose
 * error estimate exceeds `tolerance` is recomputed in FP64
 * (tbtkkpm_ldos_sites, or tbtkkpm_moments_batched + tbtkkpm_greens, at
 * TBTKKPM_FP64).  Each result depends only on its own request: the same
 * bits alone or among any other requests.  Lane memory (vectors, moments)
 * of a model is allocated when it first gets a request and counts against
 * `hbm_budget` (bytes); idle models are evicted least recently used first;
 * a request whose model does not fit waits.  Any thread may submit and
 * wait; one worker thread per server drives the device. */

typedef struct tbtkkpm_server tbtkkpm_server;

#define TBTKKPM_PENDING 1  /* tbtkkpm_server_wait: not finished yet */

/* energies[E]: the energy grid of every result (inside (-s, s) of every
 * model).  max_moments: the largest M a request may ask for.  tick_steps:
 * recursion steps between admission points (0: 64).  tolerance <= 0 never
 * recomputes. */
TBTKKPM_API int tbtkkpm_server_create(
	uint32_t max_moments, const double *energies, uint32_t E,
	uint64_t hbm_budget, uint32_t tick_steps, double tolerance,
	tbtkkpm_server **out);

/* Registers a model from its CSR (as tbtkkpm_matrix_create_csr) with
 * `width` lanes (1, 2, 4, ..., 64): a request of the model takes up to
 * `width` of them, and the lane memory (two [N][width] vector buffers, moment
 * rows) counts `width` lanes against the HBM budget.  The model id is
 * returned in *model. */
TBTKKPM_API int tbtkkpm_server_add_model(
	tbtkkpm_server *s, const uint32_t *rowptr, const uint32_t *col,
	const double *val, uint32_t N, double scale, uint32_t width,
	uint32_t *model);

/* Queues the LDOS of n_sites sites of a model (1 <= n_sites <= width,
 * 2 <= M <= max_moments); *request identifies it. */
TBTKKPM_API int tbtkkpm_server_submit(
	tbtkkpm_server *s, uint32_t model, const uint32_t *sites,
	uint32_t n_sites, uint32_t M, double broadening, uint64_t *request);

/* Queues the Green's functions G(to[k], from[k]) of one type (TBTKKPM_*
 * type codes) for n_pairs pairs of a model (calculateGreensFunction(s),
 * Lib/src/PropertyExtractor/ChebyshevExpander.cpp:96-295: coefficients
 * <to|T_n|from> of the recursion started at `from`, then
 * generateGreensFunction of that type,
 * Lib/src/Solver/ChebyshevExpander.cpp:277-361).  Pairs with the same
 * from-index share one lane; 1 <= n_pairs <= width.  If every pair has
 * to == from the lanes run the doubling recursion to M/2 as LDOS requests
 * do; otherwise they run M - 1 steps and gather every moment directly. */
TBTKKPM_API int tbtkkpm_server_submit_greens(
	tbtkkpm_server *s, uint32_t model, const uint32_t *to,
	const uint32_t *from, uint32_t n_pairs, uint32_t M, double broadening,
	int type, uint64_t *request);

/* Waits up to timeout_s seconds (0: poll) for an LDOS request.  Returns
 * TBTKKPM_OK with ldos_out [n_sites][E], err_out [n_sites] (error estimate
 * of the mixed-precision run) and rerun_out [n_sites] (1 where the FP64
 * recomputation replaced it) filled and the request released, or
 * TBTKKPM_PENDING.  Output pointers may be NULL.  A cancelled request
 * returns TBTKKPM_ERR_CANCELLED and is released. */
TBTKKPM_API int tbtkkpm_server_wait(
	tbtkkpm_server *s, uint64_t request, double timeout_s, double *ldos_out,
	double *err_out, int32_t *rerun_out);

/* Same for a Green's-function request: G_out [n_pairs][E] complex, err_out
 * and rerun_out [n_pairs].  The estimate of a pair gathered directly is its
 * source's doubling gap (the error scale of moments from the same float
 * vectors) relative to the pair's largest moment. */
TBTKKPM_API int tbtkkpm_server_wait_greens(
	tbtkkpm_server *s, uint64_t request, double timeout_s, double *G_out,
	double *err_out, int32_t *rerun_out);

/* Cancels a request that is queued or in its recursion: a queued one never
 * starts, one in flight leaves its lanes at the next step boundary; its
 * wait then returns TBTKKPM_ERR_CANCELLED.  A request whose recursion has
 * ended (its results are being formed or are ready) is not affected:
 * TBTKKPM_ERR_STATE.  Cancelling twice is not an error.  (No reference
 * counterpart.) */
TBTKKPM_API int tbtkkpm_server_cancel(tbtkkpm_server *s, uint64_t request);

/* Statistics into out[n] (n <= TBTKKPM_STAT_COUNT): */
#define TBTKKPM_STAT_COMPLETED 0  /* requests finished */
#define TBTKKPM_STAT_P50_MS 1     /* median submit-to-finish latency */
#define TBTKKPM_STAT_P99_MS 2     /* 99th percentile latency */
#define TBTKKPM_STAT_MEAN_MS 3
#define TBTKKPM_STAT_RERUNS 4     /* sites recomputed in FP64 */
#define TBTKKPM_STAT_TICKS 5
#define TBTKKPM_STAT_STEPS 6      /* recursion steps launched */
#define TBTKKPM_STAT_LANE_STEPS 7 /* sum over requests of sites * steps */
#define TBTKKPM_STAT_RESIDENT 8   /* lane bytes resident now */
#define TBTKKPM_STAT_EVICTIONS 9
#define TBTKKPM_STAT_WAITED 10    /* admissions deferred by the budget */
#define TBTKKPM_STAT_BUSY_S 11    /* worker time with lanes in flight */
#define TBTKKPM_STAT_STEP_S 12    /* device time of the recursion steps */
#define TBTKKPM_STAT_STEP_BYTES 13 /* algorithmic bytes of those steps */
#define TBTKKPM_STAT_FINISH_S 14  /* worker time in energy sums and results */
#define TBTKKPM_STAT_RERUN_S 15   /* of which FP64 recomputations */
#define TBTKKPM_STAT_JOIN_S 16    /* worker time starting lanes (FP64 heads included) */
#define TBTKKPM_STAT_PLAN_S 17    /* worker time admitting requests and planning ticks */
#define TBTKKPM_STAT_TICK_S 18    /* worker time launching ticks and waiting for them */
#define TBTKKPM_STAT_GRAPH_TICKS 19 /* ticks whose steps replayed a captured CUDA graph */
#define TBTKKPM_STAT_RELAYOUTS 20 /* step-width changes of models with lanes in flight */
#define TBTKKPM_STAT_COUNT 21
TBTKKPM_API int tbtkkpm_server_stats(tbtkkpm_server *s, double *out, uint32_t n);

/* Times every compiled step configuration of lane width `width` for
 * probe_steps steps, for each lane class (real float lanes, complex64
 * lanes) with a model of that width, on the largest model of the class
 * (the server must be idle), and keeps the fastest per class; the outputs
 * describe the class of the largest model.  With adaptive widths
 * (tbtkkpm_server_set_adaptive_width) the narrower widths down to 4 that
 * these models step at are tuned the same way.  For a tile-staged pick it
 * also builds the gather plans of every model of the class, so the first
 * tick does not.  set_config installs a known one.  Results do not depend
 * on the configuration. */
TBTKKPM_API int tbtkkpm_server_autotune(
	tbtkkpm_server *s, uint32_t width, uint32_t probe_steps, int *tpr,
	int *vpt, int *minb, double *ms_per_step);
TBTKKPM_API int tbtkkpm_server_set_config(
	tbtkkpm_server *s, uint32_t width, int tpr, int vpt, int minb);

/* Lists the compiled step configurations of lane width `width` for real
 * float lanes (real != 0) or complex64 lanes as (tpr, vpt, variant) triples
 * into out[3*cap]; returns their number.  variant 1-2 is the register cap
 * of a register-staged step; 100000 + 1000000*CV + 1000*R + 10*CW + BPS a
 * tile-staged step (rows of R-row tiles staged in shared memory by bulk
 * copies, CW consumer warps, BPS blocks per SM, CV the split of the
 * float -> FP64 widenings between the integer and conversion pipes; real
 * widths from 4, complex widths from 2).  Any of them gives the same
 * results. */
TBTKKPM_API int tbtkkpm_server_step_configs(int real, uint32_t width, int *out, int cap);

/* Models added after set_real(s, 0) keep complex64 lanes even when their
 * Hamiltonian is real; by default (1) a real model's lanes hold real float
 * vectors (tbtkkpm_matrix_set_real), with the same results. */
TBTKKPM_API int tbtkkpm_server_set_real(tbtkkpm_server *s, int enable);

/* FP64 head steps of the lanes of models added later (default 32, 0 = off;
 * tbtkkpm_matrix_set_fp64_head).  A lane's head depends only on its model,
 * site and M, so its result is the same alone and in any mix. */
TBTKKPM_API int tbtkkpm_server_set_fp64_head(tbtkkpm_server *s, uint32_t steps);

/* Scales first used after set_table_free(s, 1) get table-free energy sums
 * (tbtkkpm_table_create_clenshaw): 8 E bytes per scale instead of the
 * max_moments x E table of 16-byte entries, same results up to rounding. */
TBTKKPM_API int tbtkkpm_server_set_table_free(tbtkkpm_server *s, int enable);

/* The steps of a tick replay a CUDA graph of one step of every lane class,
 * captured when the tick starts (enable = 1, the default; a device counter
 * gives each replay its step); enable = 0 launches every kernel of every
 * step directly.  A capture that fails turns graphs off for the server.
 * Results do not depend on it.  (No reference counterpart.) */
TBTKKPM_API int tbtkkpm_server_set_graphs(tbtkkpm_server *s, int enable);

/* enable = 1 (the default): a model steps at the narrowest width (a power
 * of two, at least 4 or its lane count) that covers its highest busy lane,
 * so a step moves the vectors of those lanes only, not of all `width`
 * lanes; a request takes the lowest free lanes, and at a step boundary
 * where the width changes the model's two vector buffers are restrided in
 * place (TBTKKPM_STAT_RELAYOUTS counts these).  A step runs the
 * configuration of the width it steps at (tbtkkpm_server_set_config and
 * tbtkkpm_server_autotune set one per width).  enable = 0: every model
 * steps at its full lane count.  Results do not depend on it.  (No
 * reference counterpart.) */
TBTKKPM_API int tbtkkpm_server_set_adaptive_width(tbtkkpm_server *s, int enable);

/* Bound of each wait of the server's tile-staged steps for rows staged in
 * shared memory (polls; TBTKKPM_WAIT_DEFAULT: the library's bound), as
 * tbtkkpm_matrix_set_wait_limit.  A wait that runs out ends that step early
 * and fails every request of the server with TBTKKPM_ERR_TIMEOUT; the
 * device context stays usable.  polls = 0 makes every such wait give up at
 * once, which tests that path.  (No reference counterpart.) */
TBTKKPM_API int tbtkkpm_server_set_wait_limit(tbtkkpm_server *s, uint32_t polls);

/* Stops the worker (requests still queued or in flight are dropped) and
 * frees the server. */
TBTKKPM_API int tbtkkpm_server_destroy(tbtkkpm_server *s);

#ifdef __cplusplus
}
#endif

#endif
