/* TEST INFRASTRUCTURE ONLY — the CPU oracle of the KPM (Chebyshev) path.
 *
 * A plain-C restatement of TBTK's CPU Chebyshev expander, used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
 * The product never links or calls it.
 *
 * Pinned against: the TBTK reference compiled from its own sources
 * (oracle/_ref, built by oracle/Makefile) bit-for-bit on golden vectors
 * (tests/golden), and the closed-form known answers of the reference tests
 * (Test/include/TBTK/Test/Solver/ChebyshevExpander.h:184-564).
 *
 * Complex numbers are interleaved (re, im) doubles.  Floating-point
 * operations follow the reference's order one for one and the file is
 * compiled without FMA contraction, so results are bit-identical to the
 * reference built with the same compiler.
 */
#ifndef KPM_ORACLE_H
#define KPM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Triplets (row = basis(to), col = basis(from), value) -> CSR with columns
 * ascending in each row and duplicates summed.  rowptr has num_rows+1
 * entries, num_rows = max row + 1 (dynamic dimensions).  col/val must hold
 * n entries.  Returns the merged nnz.
 * Follows SparseMatrix::constructCSX / sortLIL / mergeLIL
 * (Lib/include/Utilities/TBTK/SparseMatrix.h:1375-1551). */
int64_t kpm_csr_from_triplets(
	int64_t n, const uint32_t *rows, const uint32_t *cols, const double *vals,
	uint32_t *rowptr, uint32_t *col, double *val, uint32_t *num_rows);

/* Chebyshev moments mu[k][n] = <to_k| T_n(H/s) |from>, n = 0..M-1, without
 * damping.  out is [K][M] complex.  Follows calculateCoefficientsCPU
 * (Lib/src/Solver/ChebyshevExpander.cpp:103-188). */
int kpm_moments(
	uint32_t N, const uint32_t *rowptr, const uint32_t *col, const double *val,
	double scale, int M, uint32_t from, int K, const uint32_t *to,
	double *out);

/* Lorentz damping in place: mu_n *= sinh(lambda(1-n/M))/sinh(lambda),
 * lambda = broadening*M; nothing when broadening == 0.
 * (Lib/src/Solver/ChebyshevExpander.cpp:190-196) */
void kpm_damp(int K, int M, double broadening, double *mu);

/* Lookup table T[n][e], [M][E] complex.
 * (Lib/src/Solver/ChebyshevExpander.cpp:201-270) */
void kpm_lookup_table(
	int M, int E, const double *energies, double scale, double *table);

/* Green's function from M coefficients over E energies.
 * type: 0 Advanced, 1 Retarded, 2 Principal, 3 NonPrincipal
 * (Solver::ChebyshevExpander::Type, ChebyshevExpander.h:203-208).
 * With a table: Lib/src/Solver/ChebyshevExpander.cpp:324-370;
 * without (closed form): :371-432.  out is [E] complex. */
void kpm_greens_table(
	int M, int E, const double *table, int type, const double *coeff,
	double *out);
void kpm_greens_closed(
	int M, int E, const double *energies, double scale, int type,
	const double *coeff, double *out);

/* LDOS[e] = Im(G_NonPrincipal[e]) / pi from a table
 * (Lib/src/PropertyExtractor/ChebyshevExpander.cpp:661-684). */
void kpm_ldos_table(
	int M, int E, const double *table, const double *coeff, double *out);

/* Energies of TBTK's Range(lower, upper, res, incl_lo, incl_hi)
 * (Lib/src/Utilities/Range.cpp:30-57, Range.h:107-109). */
void kpm_range(
	double lower, double upper, int res, int incl_lo, int incl_hi,
	double *out);

#ifdef __cplusplus
}
#endif

#endif
