/* Test infrastructure only: a C entry layer over the UNMODIFIED TBTK reference
 * classes (Model, Solver::ChebyshevExpander, PropertyExtractor::ChebyshevExpander),
 * compiled against the reference sources by oracle/Makefile into oracle/_ref/.
 * It is the checker the restatement in kpm_oracle.c is pinned against, and the
 * CPU baseline the benchmark times.  Nothing in the product links it.
 *
 * Reference call sites it drives:
 *   Model / HoppingAmplitude input      Lib/include/Core/TBTK/Model.h:430-466
 *   HoppingAmplitudeSet::getSparseMatrix Lib/include/Core/TBTK/HoppingAmplitudeSet.h:397-424
 *   Solver::ChebyshevExpander           Lib/src/Solver/ChebyshevExpander.cpp:103-435
 *   PropertyExtractor::calculateLDOS    Lib/src/PropertyExtractor/ChebyshevExpander.cpp:475-505
 *   spin-polarized LDOS, density, magnetization, expectation values
 *                                       Lib/src/PropertyExtractor/ChebyshevExpander.cpp:297-720
 */
#include "TBTK/Functions.h"
#include "TBTK/Model.h"
#include "TBTK/Property/Density.h"
#include "TBTK/Property/EnergyResolvedProperty.h"
#include "TBTK/Property/GreensFunction.h"
#include "TBTK/Property/LDOS.h"
#include "TBTK/PropertyExtractor/ChebyshevExpander.h"
#include "TBTK/Range.h"
#include "TBTK/Solver/ChebyshevExpander.h"
#include "TBTK/Streams.h"
#include "TBTK/TBTK.h"

#include <algorithm>
#include <complex>
#include <cstdint>
#include <string>
#include <vector>

using namespace TBTK;
using cplx = std::complex<double>;

namespace {

Index make_index(const int *p, int len){
	Index idx;
	for(int k = 0; k < len; k++)
		idx.pushBack(p[k]);
	return idx;
}

Solver::ChebyshevExpander::Type to_type(int type){
	switch(type){
	case 0: return Solver::ChebyshevExpander::Type::Advanced;
	case 1: return Solver::ChebyshevExpander::Type::Retarded;
	case 2: return Solver::ChebyshevExpander::Type::Principal;
	default: return Solver::ChebyshevExpander::Type::NonPrincipal;
	}
}

struct Quiet{
	Quiet(){
		Communicator::setGlobalVerbose(false);
		//Units and constants (the occupation functions need k_B).
		TBTK::Initialize();
	}
} quiet;

} // namespace

extern "C" {

/* Builds and constructs a Model from explicit amplitudes: amplitude k is
 * amp[2k] + i amp[2k+1], from index from_idx[k*idx_len ...] to index
 * to_idx[k*idx_len ...].  No Hermitian conjugate is added implicitly. */
void *ref_model_create(
	int64_t n_amp, int idx_len, const int *to_idx, const int *from_idx,
	const double *amp
){
	Model *model = new Model();
	model->setVerbose(false);
	for(int64_t k = 0; k < n_amp; k++){
		*model << HoppingAmplitude(
			cplx(amp[2*k], amp[2*k + 1]),
			make_index(to_idx + k*idx_len, idx_len),
			make_index(from_idx + k*idx_len, idx_len)
		);
	}
	model->construct();
	return model;
}

void ref_model_destroy(void *model){
	delete (Model*)model;
}

int ref_model_basis_size(void *model){
	return ((Model*)model)->getBasisSize();
}

int ref_model_basis_index(void *model, const int *idx, int idx_len){
	return ((Model*)model)->getBasisIndex(make_index(idx, idx_len));
}

/* CSR of getSparseMatrix() after setStorageFormat(CSR), exactly as
 * calculateCoefficientsCPU sees it before scaling.  Returns nnz, or -nnz-1
 * when cap is too small (nothing written then). */
int64_t ref_model_csr(
	void *model, uint32_t *rowptr, uint32_t *col, double *val, int64_t cap,
	int *num_rows
){
	const HoppingAmplitudeSet &has
		= ((Model*)model)->getHoppingAmplitudeSet();
	SparseMatrix<cplx> sm = has.getSparseMatrix();
	sm.setStorageFormat(SparseMatrix<cplx>::StorageFormat::CSR);
	const unsigned int nr = sm.getNumRows();
	const unsigned int *rp = sm.getCSRRowPointers();
	const int64_t nnz = rp[nr];
	*num_rows = (int)nr;
	if(nnz > cap)
		return -nnz - 1;
	const unsigned int *c = sm.getCSRColumns();
	const cplx *v = sm.getCSRValues();
	for(unsigned int r = 0; r <= nr; r++)
		rowptr[r] = rp[r];
	for(int64_t k = 0; k < nnz; k++){
		col[k] = c[k];
		val[2*k] = v[k].real();
		val[2*k + 1] = v[k].imag();
	}
	return nnz;
}

/* Solver::ChebyshevExpander::calculateCoefficients (CPU) for K to-indices
 * and one from-index.  out is [K][M][2]. */
int ref_coefficients(
	void *model, double scale, int M, double broadening,
	int K, int idx_len, const int *to, const int *from, double *out
){
	Solver::ChebyshevExpander solver;
	solver.setVerbose(false);
	solver.setModel(*(Model*)model);
	solver.setScaleFactor(scale);
	solver.setNumCoefficients(M);
	solver.setBroadening(broadening);
	solver.setCalculateCoefficientsOnGPU(false);
	std::vector<Index> tos;
	for(int k = 0; k < K; k++)
		tos.push_back(make_index(to + k*idx_len, idx_len));
	std::vector<std::vector<cplx>> c = solver.calculateCoefficients(
		tos, make_index(from, idx_len)
	);
	for(int k = 0; k < K; k++){
		for(int n = 0; n < M; n++){
			out[2*((int64_t)k*M + n)] = c[k][n].real();
			out[2*((int64_t)k*M + n) + 1] = c[k][n].imag();
		}
	}
	return 0;
}

/* Energy k of Range(lower, upper, res, incl_lo, incl_hi). */
double ref_range_value(
	double lower, double upper, int res, int incl_lo, int incl_hi, int k
){
	Range r(lower, upper, res, incl_lo != 0, incl_hi != 0);
	return r[k];
}

/* Solver::ChebyshevExpander::generateGreensFunction (CPU) for one
 * coefficient vector of length M.  type: 0 Advanced, 1 Retarded,
 * 2 Principal, 3 NonPrincipal.  out is [res][2]. */
int ref_greens(
	double scale, int M, double lower, double upper, int res, int incl_lo,
	int incl_hi, int use_table, int type, const double *coeff, double *out
){
	Solver::ChebyshevExpander solver;
	solver.setVerbose(false);
	solver.setScaleFactor(scale);
	solver.setNumCoefficients(M);
	solver.setGenerateGreensFunctionsOnGPU(false);
	solver.setUseLookupTable(use_table != 0);
	solver.setEnergyWindow(
		Range(lower, upper, res, incl_lo != 0, incl_hi != 0)
	);
	std::vector<cplx> c(M);
	for(int n = 0; n < M; n++)
		c[n] = cplx(coeff[2*n], coeff[2*n + 1]);
	std::vector<cplx> g = solver.generateGreensFunction(c, to_type(type));
	for(int e = 0; e < res; e++){
		out[2*e] = g[e].real();
		out[2*e + 1] = g[e].imag();
	}
	return 0;
}

/* PropertyExtractor::ChebyshevExpander::calculateLDOS({sites}) with the
 * PropertyExtractor's inclusive window Range(lower, upper, res).
 * use_table selects Solver::setUseLookupTable.  out is [n_sites][res]. */
int ref_ldos(
	void *model, double scale, int M, double broadening, double lower,
	double upper, int res, int use_table, int n_sites, int idx_len,
	const int *sites, double *out
){
	Solver::ChebyshevExpander solver;
	solver.setVerbose(false);
	solver.setModel(*(Model*)model);
	solver.setScaleFactor(scale);
	solver.setNumCoefficients(M);
	solver.setBroadening(broadening);
	solver.setUseLookupTable(use_table != 0);
	PropertyExtractor::ChebyshevExpander pe(solver);
	pe.setEnergyWindow(lower, upper, res);
	std::vector<Index> patterns;
	for(int k = 0; k < n_sites; k++)
		patterns.push_back(make_index(sites + k*idx_len, idx_len));
	Property::LDOS ldos = pe.calculateLDOS(patterns);
	for(int k = 0; k < n_sites; k++){
		Index site = make_index(sites + k*idx_len, idx_len);
		for(int e = 0; e < res; e++)
			out[(int64_t)k*res + e] = ldos(site, e);
	}
	return 0;
}

/* PropertyExtractor::ChebyshevExpander::calculateGreensFunctions(to, from)
 * with the PropertyExtractor's inclusive window.  out is [K][res][2]. */
int ref_greens_pe(
	void *model, double scale, int M, double broadening, double lower,
	double upper, int res, int use_table, int type, int K, int idx_len,
	const int *to, const int *from, double *out
){
	Solver::ChebyshevExpander solver;
	solver.setVerbose(false);
	solver.setModel(*(Model*)model);
	solver.setScaleFactor(scale);
	solver.setNumCoefficients(M);
	solver.setBroadening(broadening);
	solver.setUseLookupTable(use_table != 0);
	PropertyExtractor::ChebyshevExpander pe(solver);
	pe.setEnergyWindow(lower, upper, res);
	/* calculateGreensFunctions generates G for its to-indices inside an
	 * OpenMP loop (PropertyExtractor/ChebyshevExpander.cpp:278-292) whose
	 * first iterations race on the lazy lookup-table build
	 * (Solver/ChebyshevExpander.h:548-566); one serial call builds the
	 * table first. */
	solver.generateGreensFunction(
		std::vector<cplx>(M, cplx(0, 0)),
		Solver::ChebyshevExpander::Type::Retarded
	);
	std::vector<Index> tos;
	for(int k = 0; k < K; k++)
		tos.push_back(make_index(to + k*idx_len, idx_len));
	Index f = make_index(from, idx_len);
	Property::GreensFunction::Type t;
	switch(type){
	case 0: t = Property::GreensFunction::Type::Advanced; break;
	case 1: t = Property::GreensFunction::Type::Retarded; break;
	case 2: t = Property::GreensFunction::Type::Principal; break;
	default: t = Property::GreensFunction::Type::NonPrincipal; break;
	}
	Property::GreensFunction gf = pe.calculateGreensFunctions(tos, f, t);
	for(int k = 0; k < K; k++){
		for(int e = 0; e < res; e++){
			cplx v = gf({tos[k], f}, e);
			out[2*((int64_t)k*res + e)] = v.real();
			out[2*((int64_t)k*res + e) + 1] = v.imag();
		}
	}
	return 0;
}


/* One site of PropertyExtractor::ChebyshevExpander's other properties,
 * with the model at temperature T and chemical potential mu and the
 * PropertyExtractor's inclusive window Range(lower, upper, res).  The site
 * is `index` (idx_len entries); an entry -1 marks the spin subindex
 * (IDX_SPIN).  kind 0: calculateSpinPolarizedLDOS, out [res][2][2][2]
 * (complex (a, b) entries); kind 1: calculateDensity, out [1]; kind 2:
 * calculateMagnetization, out [2][2][2]. */
int ref_property(
	void *model, double scale, int M, double broadening, double lower,
	double upper, int res, int use_table, double T, double mu, int kind,
	int idx_len, const int *index, double *out
){
	Model &mdl = *(Model*)model;
	mdl.setTemperature(T);
	mdl.setChemicalPotential(mu);
	Solver::ChebyshevExpander solver;
	solver.setVerbose(false);
	solver.setModel(mdl);
	solver.setScaleFactor(scale);
	solver.setNumCoefficients(M);
	solver.setBroadening(broadening);
	solver.setUseLookupTable(use_table != 0);
	PropertyExtractor::ChebyshevExpander pe(solver);
	pe.setEnergyWindow(lower, upper, res);
	Index pattern;
	for(int k = 0; k < idx_len; k++)
		pattern.pushBack(index[k] == -1 ? (int)IDX_SPIN : index[k]);
	auto put = [&](const SpinMatrix &s, double *o){
		for(int a = 0; a < 2; a++){
			for(int b = 0; b < 2; b++){
				o[2*(2*a + b)] = s.at(a, b).real();
				o[2*(2*a + b) + 1] = s.at(a, b).imag();
			}
		}
	};
	if(kind == 0){
		Property::SpinPolarizedLDOS p
			= pe.calculateSpinPolarizedLDOS({pattern});
		const std::vector<SpinMatrix> &d = p.getData();
		for(int e = 0; e < res && e < (int)d.size(); e++)
			put(d[e], out + 8*(int64_t)e);
		return (int)d.size();
	}
	if(kind == 1){
		Property::Density p = pe.calculateDensity({pattern});
		out[0] = p.getData()[0];
		return (int)p.getData().size();
	}
	Property::Magnetization p = pe.calculateMagnetization({pattern});
	put(p.getData()[0], out);
	return (int)p.getData().size();
}

/* PropertyExtractor::ChebyshevExpander::calculateExpectationValue(to, from)
 * at temperature T and chemical potential mu; out [2]. */
int ref_expectation(
	void *model, double scale, int M, double broadening, double lower,
	double upper, int res, int use_table, double T, double mu, int idx_len,
	const int *to, const int *from, double *out
){
	Model &mdl = *(Model*)model;
	mdl.setTemperature(T);
	mdl.setChemicalPotential(mu);
	Solver::ChebyshevExpander solver;
	solver.setVerbose(false);
	solver.setModel(mdl);
	solver.setScaleFactor(scale);
	solver.setNumCoefficients(M);
	solver.setBroadening(broadening);
	solver.setUseLookupTable(use_table != 0);
	PropertyExtractor::ChebyshevExpander pe(solver);
	pe.setEnergyWindow(lower, upper, res);
	cplx v = pe.calculateExpectationValue(
		make_index(to, idx_len), make_index(from, idx_len)
	);
	out[0] = v.real();
	out[1] = v.imag();
	return 0;
}

/* Functions::fermiDiracDistribution(energy, mu, T), the occupation the
 * properties above weight with (PropertyExtractor.h:910-935). */
double ref_fermi_dirac(double energy, double mu, double T){
	return Functions::fermiDiracDistribution(energy, mu, T);
}

} // extern "C"

namespace {

/* Copies s with a terminating 0 into out when it fits in cap bytes. */
int64_t put_string(const std::string &s, char *out, int64_t cap){
	if(out != nullptr && (int64_t)s.size() < cap){
		std::copy(s.begin(), s.end(), out);
		out[s.size()] = 0;
	}
	return (int64_t)s.size();
}

template<typename DataType>
void put_data(const std::vector<DataType> &d, double *values, int64_t cap);

template<>
void put_data(const std::vector<double> &d, double *values, int64_t cap){
	for(int64_t n = 0; n < (int64_t)d.size() && n < cap; n++)
		values[n] = d[n];
}

template<>
void put_data(const std::vector<cplx> &d, double *values, int64_t cap){
	for(int64_t n = 0; n < (int64_t)d.size() && 2*n + 1 < cap; n++){
		values[2*n] = d[n].real();
		values[2*n + 1] = d[n].imag();
	}
}

} // namespace

extern "C" {

/* A property computed by the reference and its JSON serialization
 * (Serializable::Mode::JSON):
 *   kind 0: PropertyExtractor::calculateLDOS(sites) -> Property::LDOS
 *           (Lib/src/Property/LDOS.cpp:121-140);
 *   kind 1: calculateGreensFunctions(sites, from, type) ->
 *           Property::GreensFunction, written by its EnergyResolvedProperty
 *           base (Lib/include/TBTK/Property/EnergyResolvedProperty.h:1156-1212);
 *   kind 2: calculateDensity(sites) at temperature T and chemical potential
 *           mu -> Property::Density (Lib/src/Property/Density.cpp:111-130).
 * The property's data array goes to values (complex data as (re, im)
 * pairs, at most values_cap doubles).  Returns the length of the JSON text,
 * written with a terminating 0 into out when it fits in cap bytes. */
int64_t ref_property_json(
	void *model, double scale, int M, double broadening, double lower,
	double upper, int res, int use_table, double T, double mu, int kind,
	int type, int n_sites, int idx_len, const int *sites, const int *from,
	char *out, int64_t cap, double *values, int64_t values_cap
){
	Model &mdl = *(Model*)model;
	mdl.setTemperature(T);
	mdl.setChemicalPotential(mu);
	Solver::ChebyshevExpander solver;
	solver.setVerbose(false);
	solver.setModel(mdl);
	solver.setScaleFactor(scale);
	solver.setNumCoefficients(M);
	solver.setBroadening(broadening);
	solver.setUseLookupTable(use_table != 0);
	PropertyExtractor::ChebyshevExpander pe(solver);
	pe.setEnergyWindow(lower, upper, res);
	std::vector<Index> patterns;
	for(int k = 0; k < n_sites; k++)
		patterns.push_back(make_index(sites + k*idx_len, idx_len));
	if(kind == 0){
		Property::LDOS p = pe.calculateLDOS(patterns);
		put_data(p.getData(), values, values_cap);
		return put_string(p.serialize(Serializable::Mode::JSON), out, cap);
	}
	if(kind == 1){
		/* one serial table build first: calculateGreensFunctions races on
		 * the lazy build (see ref_greens_pe) */
		solver.generateGreensFunction(
			std::vector<cplx>(M, cplx(0, 0)),
			Solver::ChebyshevExpander::Type::Retarded
		);
		Property::GreensFunction::Type t;
		switch(type){
		case 0: t = Property::GreensFunction::Type::Advanced; break;
		case 1: t = Property::GreensFunction::Type::Retarded; break;
		case 2: t = Property::GreensFunction::Type::Principal; break;
		default: t = Property::GreensFunction::Type::NonPrincipal; break;
		}
		Property::GreensFunction p = pe.calculateGreensFunctions(
			patterns, make_index(from, idx_len), t
		);
		put_data(p.getData(), values, values_cap);
		return put_string(p.serialize(Serializable::Mode::JSON), out, cap);
	}
	Property::Density p = pe.calculateDensity(patterns);
	put_data(p.getData(), values, values_cap);
	return put_string(p.serialize(Serializable::Mode::JSON), out, cap);
}

/* Reads a serialization with the reference's deserializing constructor
 * (kind 0 Property::LDOS, kind 1 EnergyResolvedProperty<complex<double>>,
 * kind 2 Property::Density) and serializes the object again; the data
 * array read goes to values as in ref_property_json.  Returns the length
 * of the new serialization, written into out as above.  A text the
 * reference cannot parse ends the process with TBTKExit's exit(1). */
int64_t ref_json_reserialize(
	int kind, const char *json, char *out, int64_t cap, double *values,
	int64_t values_cap
){
	const std::string s(json);
	if(kind == 0){
		Property::LDOS p(s, Serializable::Mode::JSON);
		put_data(p.getData(), values, values_cap);
		return put_string(p.serialize(Serializable::Mode::JSON), out, cap);
	}
	if(kind == 1){
		Property::EnergyResolvedProperty<cplx> p(s, Serializable::Mode::JSON);
		put_data(p.getData(), values, values_cap);
		return put_string(p.serialize(Serializable::Mode::JSON), out, cap);
	}
	Property::Density p(s, Serializable::Mode::JSON);
	put_data(p.getData(), values, values_cap);
	return put_string(p.serialize(Serializable::Mode::JSON), out, cap);
}

}
