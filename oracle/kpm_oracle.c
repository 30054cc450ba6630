/* TEST INFRASTRUCTURE ONLY — CPU oracle of the KPM path (see kpm_oracle.h).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * Each function restates one piece of TBTK's CPU Chebyshev expander; the
 * reference file:line is given beside it.  Complex products are written out
 * as (ac - bd, ad + bc), which is what GCC emits for std::complex<double>
 * (with the NaN fallback that finite inputs never reach).
 */
#pragma GCC optimize("fp-contract=off")

#include "kpm_oracle.h"

#define _GNU_SOURCE
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cx;

static inline cx cmul(cx a, cx b){
	cx r;
	r.re = a.re*b.re - a.im*b.im;
	r.im = a.re*b.im + a.im*b.re;
	return r;
}

/* ------------------------------------------------------------ matrix */

typedef struct { uint32_t row, col; int64_t order; } key_t_;

static int key_cmp(const void *pa, const void *pb){
	const key_t_ *a = (const key_t_*)pa, *b = (const key_t_*)pb;
	if(a->row != b->row) return a->row < b->row ? -1 : 1;
	if(a->col != b->col) return a->col < b->col ? -1 : 1;
	/* Duplicates keep insertion order: the reference's per-list sort is an
	 * insertion sort for the short lists of a tight-binding row
	 * (SparseMatrix.h:1375-1390). */
	return a->order < b->order ? -1 : (a->order > b->order);
}

/* SparseMatrix::constructCSX (SparseMatrix.h:1417-1551) with sortLIL
 * (:1375-1390) and mergeLIL (:1393-1414).  mergeLIL walks each list from
 * the back and folds entry y into y-1, so duplicates d0,d1,d2 sum as
 * d0 + (d1 + d2). */
int64_t kpm_csr_from_triplets(
	int64_t n, const uint32_t *rows, const uint32_t *cols, const double *vals,
	uint32_t *rowptr, uint32_t *col, double *val, uint32_t *num_rows
){
	key_t_ *keys = (key_t_*)malloc(sizeof(key_t_)*(size_t)(n > 0 ? n : 1));
	uint32_t nr = 0;
	for(int64_t k = 0; k < n; k++){
		keys[k].row = rows[k];
		keys[k].col = cols[k];
		keys[k].order = k;
		if(rows[k] + 1 > nr)
			nr = rows[k] + 1;
	}
	qsort(keys, (size_t)n, sizeof(key_t_), key_cmp);
	int64_t out = 0;
	int64_t k = 0;
	for(uint32_t r = 0; r <= nr; r++)
		rowptr[r] = 0;
	while(k < n){
		int64_t e = k;
		while(e + 1 < n && keys[e + 1].row == keys[k].row
			&& keys[e + 1].col == keys[k].col)
			e++;
		/* fold from the back */
		double re = vals[2*keys[e].order], im = vals[2*keys[e].order + 1];
		for(int64_t y = e - 1; y >= k; y--){
			re = vals[2*keys[y].order] + re;
			im = vals[2*keys[y].order + 1] + im;
		}
		col[out] = keys[k].col;
		val[2*out] = re;
		val[2*out + 1] = im;
		rowptr[keys[k].row + 1]++;
		out++;
		k = e + 1;
	}
	for(uint32_t r = 0; r < nr; r++)
		rowptr[r + 1] += rowptr[r];
	*num_rows = nr;
	free(keys);
	return out;
}

/* ------------------------------------------------------------ moments */

/* addHamiltonianProduct (ChebyshevExpander.cpp:65-82): result[row] +=
 * values[n]*vector[col[n]] in ascending n. */
static void add_product(
	uint32_t nrows, const uint32_t *rowptr, const uint32_t *col,
	const cx *v, const cx *x, cx *y
){
	for(uint32_t r = 0; r < nrows; r++){
		for(uint32_t k = rowptr[r]; k < rowptr[r + 1]; k++){
			cx p = cmul(v[k], x[col[k]]);
			y[r].re = y[r].re + p.re;
			y[r].im = y[r].im + p.im;
		}
	}
}

/* calculateCoefficientsCPU (ChebyshevExpander.cpp:103-188).  The matrix
 * rows are min(N, rowptr rows); rows past the stored ones are empty. */
int kpm_moments(
	uint32_t N, const uint32_t *rowptr, const uint32_t *col, const double *val,
	double scale, int M, uint32_t from, int K, const uint32_t *to,
	double *out
){
	if(M <= 0 || from >= N)
		return -1;
	for(int k = 0; k < K; k++)
		if(to[k] >= N)
			return -1;
	const int64_t nnz = rowptr[N];
	cx *v = (cx*)malloc(sizeof(cx)*(size_t)(nnz > 0 ? nnz : 1));
	/* sparseMatrix *= 1/scaleFactor (:147): complex * complex(1/s, 0) */
	const cx inv = {1/scale, 0.0};
	for(int64_t k = 0; k < nnz; k++){
		cx a = {val[2*k], val[2*k + 1]};
		v[k] = cmul(a, inv);
	}
	cx *j1 = (cx*)calloc(N, sizeof(cx));
	cx *j2 = (cx*)calloc(N, sizeof(cx));
	cx *jr = (cx*)calloc(N, sizeof(cx));
	memset(out, 0, sizeof(double)*2*(size_t)K*(size_t)M);
	j1[from].re = 1.0;
	for(int k = 0; k < K; k++){
		out[2*((int64_t)k*M)] = j1[to[k]].re;
		out[2*((int64_t)k*M) + 1] = j1[to[k]].im;
	}
	/* |j1> = H~|j0> into a zeroed result (:160-164) */
	add_product(N, rowptr, col, v, j1, jr);
	{ cx *t = j2; j2 = j1; j1 = jr; jr = t; }
	if(M > 1){
		for(int k = 0; k < K; k++){
			out[2*((int64_t)k*M + 1)] = j1[to[k]].re;
			out[2*((int64_t)k*M + 1) + 1] = j1[to[k]].im;
		}
	}
	/* sparseMatrix *= 2 (:168): complex * complex(2, 0) */
	const cx two = {2.0, 0.0};
	for(int64_t k = 0; k < nnz; k++)
		v[k] = cmul(v[k], two);
	for(int n = 2; n < M; n++){
		for(uint32_t c = 0; c < N; c++){
			jr[c].re = -j2[c].re;
			jr[c].im = -j2[c].im;
		}
		add_product(N, rowptr, col, v, j1, jr);
		{ cx *t = j2; j2 = j1; j1 = jr; jr = t; }
		for(int k = 0; k < K; k++){
			out[2*((int64_t)k*M + n)] = j1[to[k]].re;
			out[2*((int64_t)k*M + n) + 1] = j1[to[k]].im;
		}
	}
	free(v); free(j1); free(j2); free(jr);
	return 0;
}

/* Lorentzian convolution (ChebyshevExpander.cpp:190-196):
 * coefficients[c][n]*sinh(lambda*(1 - n/(double)M))/sinh(lambda), i.e. a
 * complex times a real, then divided by a real, component-wise. */
void kpm_damp(int K, int M, double broadening, double *mu){
	if(broadening == 0)
		return;
	const double lambda = broadening*M;
	for(int n = 0; n < M; n++){
		const double a = sinh(lambda*(1 - n/(double)M));
		const double b = sinh(lambda);
		for(int k = 0; k < K; k++){
			double *c = mu + 2*((int64_t)k*M + n);
			c[0] = c[0]*a/b;
			c[1] = c[1]*a/b;
		}
	}
}

/* ------------------------------------------------------------ table */

/* generateLookupTable (ChebyshevExpander.cpp:258-268):
 *   (1/s) * (-2.*i/sqrt(1 - E*E)) * exp(-i*((double)n)*acos(E)) / denominator
 * evaluated left to right with std::complex semantics: real*complex and
 * complex/real are component-wise, -i is (-0, -1), exp is cexp. */
void kpm_lookup_table(
	int M, int E, const double *energies, double scale, double *table
){
	#pragma omp parallel for
	for(int n = 0; n < M; n++){
		const double denominator = n == 0 ? 2. : 1.;
		for(int e = 0; e < E; e++){
			const double x = energies[e]/scale;
			const double q = sqrt(1 - x*x);
			/* -2.*i / q */
			cx a = {-2.0*0.0, -2.0*1.0};
			a.re = a.re/q; a.im = a.im/q;
			/* (1/s) * a */
			const double is = 1/scale;
			cx b = {is*a.re, is*a.im};
			/* -i * n * acos(x) */
			const double th = acos(x);
			cx arg = {-0.0, -1.0};
			arg.re = arg.re*(double)n; arg.im = arg.im*(double)n;
			arg.re = arg.re*th; arg.im = arg.im*th;
			double complex ex = cexp(CMPLX(arg.re, arg.im));
			cx c = {creal(ex), cimag(ex)};
			cx r = cmul(b, c);
			r.re = r.re/denominator; r.im = r.im/denominator;
			table[2*((int64_t)n*E + e)] = r.re;
			table[2*((int64_t)n*E + e) + 1] = r.im;
		}
	}
}

/* ------------------------------------------------------------ Green's function */

/* generateGreensFunctionCPU with a lookup table
 * (ChebyshevExpander.cpp:324-361), n outer, e inner. */
void kpm_greens_table(
	int M, int E, const double *table, int type, const double *coeff,
	double *out
){
	memset(out, 0, sizeof(double)*2*(size_t)E);
	for(int n = 0; n < M; n++){
		const cx c = {coeff[2*n], coeff[2*n + 1]};
		for(int e = 0; e < E; e++){
			const cx t = {table[2*((int64_t)n*E + e)],
				table[2*((int64_t)n*E + e) + 1]};
			cx p;
			switch(type){
			case 1: /* Retarded: G += T*c */
				p = cmul(t, c);
				out[2*e] = out[2*e] + p.re;
				out[2*e + 1] = out[2*e + 1] + p.im;
				break;
			case 0: { /* Advanced: G += c*conj(T) */
				const cx tc = {t.re, -t.im};
				p = cmul(c, tc);
				out[2*e] = out[2*e] + p.re;
				out[2*e + 1] = out[2*e + 1] + p.im;
				break;
			}
			case 2: /* Principal: G += -c*Re(T) */
				p.re = -c.re*t.re;
				p.im = -c.im*t.re;
				out[2*e] = out[2*e] + p.re;
				out[2*e + 1] = out[2*e + 1] + p.im;
				break;
			default: { /* NonPrincipal: G -= c*i*Im(T) */
				const cx ii = {0.0, 1.0};
				cx ci = cmul(c, ii);
				p.re = ci.re*t.im;
				p.im = ci.im*t.im;
				out[2*e] = out[2*e] - p.re;
				out[2*e + 1] = out[2*e + 1] - p.im;
				break;
			}
			}
		}
	}
}

/* generateGreensFunctionCPU without a table (ChebyshevExpander.cpp:371-432). */
void kpm_greens_closed(
	int M, int E, const double *energies, double scale, int type,
	const double *coeff, double *out
){
	for(int e = 0; e < E; e++){
		cx g;
		if(type == 2){
			g.re = 0; g.im = 0;
		}
		else{
			g.re = coeff[0]/2.; g.im = coeff[1]/2.;
		}
		const double x = energies[e]/scale;
		const double th = acos(x);
		for(int n = 1; n < M; n++){
			const cx c = {coeff[2*n], coeff[2*n + 1]};
			if(type == 1 || type == 0){
				/* exp(-i*((double)n)*acosE) */
				cx arg = {-0.0, -1.0};
				arg.re = arg.re*(double)n; arg.im = arg.im*(double)n;
				arg.re = arg.re*th; arg.im = arg.im*th;
				double complex ex = cexp(CMPLX(arg.re, arg.im));
				const cx w = {creal(ex), cimag(ex)};
				cx p = cmul(c, w);
				if(type == 0)
					p.im = -p.im;
				g.re = g.re + p.re;
				g.im = g.im + p.im;
			}
			else if(type == 2){
				const double w = sin(((double)n)*th);
				g.re = g.re + c.re*w;
				g.im = g.im + c.im*w;
			}
			else{
				const double w = cos(((double)n)*th);
				g.re = g.re + c.re*w;
				g.im = g.im + c.im*w;
			}
		}
		/* *= -2.*i/s, 2.*i/s, 2./s, 2.*i/s: complex*complex except the
		 * real factor of the Principal type */
		if(type == 2){
			const double f = 2./scale;
			g.re = g.re*f; g.im = g.im*f;
		}
		else{
			cx f = {(type == 1 ? -2. : 2.)*0.0, (type == 1 ? -2. : 2.)*1.0};
			f.re = f.re/scale; f.im = f.im/scale;
			g = cmul(g, f);
		}
		const double q = sqrt(1 - x*x);
		out[2*e] = g.re/q;
		out[2*e + 1] = g.im/q;
	}
}

/* calculateLDOSCallback (PropertyExtractor/ChebyshevExpander.cpp:661-684):
 * data[e] += imag(G_NonPrincipal[e])/M_PI into a zeroed property. */
void kpm_ldos_table(
	int M, int E, const double *table, const double *coeff, double *out
){
	double *g = (double*)malloc(sizeof(double)*2*(size_t)E);
	kpm_greens_table(M, E, table, 3, coeff, g);
	for(int e = 0; e < E; e++)
		out[e] = 0.0 + g[2*e + 1]/3.14159265358979323846;
	free(g);
}

/* Range (Utilities/Range.cpp:30-57; operator[] Range.h:107-109). */
void kpm_range(
	double lower, double upper, int res, int incl_lo, int incl_hi,
	double *out
){
	double dx, start;
	if(incl_lo && incl_hi)
		dx = (upper - lower)/(res - 1);
	else if(incl_lo || incl_hi)
		dx = (upper - lower)/res;
	else
		dx = (upper - lower)/(res + 1);
	start = incl_lo ? lower : lower + dx;
	for(int k = 0; k < res; k++)
		out[k] = start + (unsigned int)k*dx;
}
