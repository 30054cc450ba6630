/* TBTK's own Solver/PropertyExtractor::ChebyshevExpander, linked against the
 * B200 seam (tbtk_b200/seam) instead of Lib/src/cuda or Lib/src/nocuda, run
 * with the reference's GPU flags and compared with the same objects on their
 * CPU path.  The same source builds two programs (tests/cpp/Makefile):
 * test_seam links the reference's PropertyExtractor::ChebyshevExpander
 * (per-index recursions), test_pe_seam links the seam's batched one
 * (tbtk_b200/seam/PropertyExtractorChebyshevExpanderB200.cpp).
 *
 *   test_seam            all parity checks; exit 0 when all pass
 *   test_seam exit-short generateGreensFunction on the GPU path with fewer
 *                        coefficients than the lookup table; must end in
 *                        TBTKExit (message on Streams::err, exit status 1)
 *   test_seam dump cpu|gpu FILE
 *                        every PropertyExtractor property of the 6x6 model
 *                        (both pattern forms) on the CPU or GPU path,
 *                        written to FILE as named blocks of doubles
 *   test_seam time       calculateLDOS of 64 sites of a 256x256 lattice with
 *                        spin through TBTK's API on the GPU path (one JSON
 *                        line: seconds, and the LDOS error of the mixed
 *                        precision against FP64)
 *
 * Expected agreement: coefficients bit-identical (the library's FP64 step
 * follows calculateCoefficientsCPU's operation order,
 * Lib/src/Solver/ChebyshevExpander.cpp:150-238); Green's functions from the
 * uploaded host lookup table bit-identical to generateGreensFunctionCPU's
 * table branch (ChebyshevExpander.cpp:371-398); LDOS therefore identical.
 */
#include "TBTK/GPUResourceManager.h"
#include "TBTK/Model.h"
#include "TBTK/PropertyExtractor/ChebyshevExpander.h"
#include "TBTK/Range.h"
#include "TBTK/Solver/ChebyshevExpander.h"
#include "TBTK/Streams.h"
#include "TBTK/TBTK.h"

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace TBTK;
using cplx = std::complex<double>;
using Type = Solver::ChebyshevExpander::Type;

namespace{

int failures = 0;

void report(const std::string &name, bool ok, const std::string &detail){
	std::printf("[%s] %s %s\n", ok ? "PASS" : "FAIL", name.c_str(),
		detail.c_str());
	if(!ok)
		failures++;
}

/* 6x6 open square lattice with spin: nearest-neighbour hopping -1, a
 * complex spin-flip hopping 0.3i on +x bonds, on-site energies from a fixed
 * integer sequence in [-0.5, 0.5]. */
void buildModel(Model &model){
	const int L = 6;
	unsigned int state = 12345u;
	auto next = [&state](){
		state = state*1103515245u + 12345u;
		return ((state >> 8) & 0xffff)/65535.0 - 0.5;
	};
	for(int x = 0; x < L; x++){
		for(int y = 0; y < L; y++){
			for(int s = 0; s < 2; s++){
				model << HoppingAmplitude(
					next(), {x, y, s}, {x, y, s}
				);
				if(x + 1 < L){
					model << HoppingAmplitude(
						-1.0, {x + 1, y, s}, {x, y, s}
					) + HC;
					model << HoppingAmplitude(
						cplx(0, 0.3), {x + 1, y, 1 - s},
						{x, y, s}
					) + HC;
				}
				if(y + 1 < L){
					model << HoppingAmplitude(
						-1.0, {x, y + 1, s}, {x, y, s}
					) + HC;
				}
			}
		}
	}
	model.construct();
}

void configure(
	Solver::ChebyshevExpander &solver, Model &model, int M, bool gpu
){
	solver.setVerbose(false);
	solver.setModel(model);
	solver.setScaleFactor(8);
	solver.setNumCoefficients(M);
	solver.setBroadening(1e-3);
	solver.setEnergyWindow(Range(-4, 4, 401, false, false));
	solver.setUseLookupTable(true);
	solver.setCalculateCoefficientsOnGPU(gpu);
	solver.setGenerateGreensFunctionsOnGPU(gpu);
}

bool sameBits(const std::vector<cplx> &a, const std::vector<cplx> &b){
	return a.size() == b.size()
		&& std::memcmp(a.data(), b.data(), a.size()*sizeof(cplx)) == 0;
}

double maxDiff(const std::vector<cplx> &a, const std::vector<cplx> &b){
	double d = a.size() == b.size() ? 0 : INFINITY;
	for(size_t n = 0; n < a.size() && n < b.size(); n++)
		d = std::fmax(d, std::abs(a[n] - b[n]));
	return d;
}

void testDevices(){
	const int n = GPUResourceManager::getInstance().getNumDevices();
	report("device_table", n >= 1, "devices=" + std::to_string(n));
}

void testCoefficients(Model &model){
	Solver::ChebyshevExpander cpu, gpu;
	configure(cpu, model, 512, false);
	configure(gpu, model, 512, true);

	std::vector<Index> to = {
		{0, 0, 0}, {0, 0, 1}, {3, 2, 0}, {5, 5, 1}, {2, 4, 1}
	};
	const Index from = {3, 2, 0};
	std::vector<std::vector<cplx>> a = cpu.calculateCoefficients(to, from);
	std::vector<std::vector<cplx>> b = gpu.calculateCoefficients(to, from);
	bool ok = a.size() == b.size();
	double d = 0;
	for(size_t k = 0; ok && k < a.size(); k++){
		ok = ok && sameBits(a[k], b[k]);
		d = std::fmax(d, maxDiff(a[k], b[k]));
	}
	report("coefficients_many_to", ok, "max|diff|=" + std::to_string(d));

	std::vector<cplx> c = cpu.calculateCoefficients({2, 4, 1}, {2, 4, 1});
	std::vector<cplx> g = gpu.calculateCoefficients({2, 4, 1}, {2, 4, 1});
	report("coefficients_single", sameBits(c, g),
		"max|diff|=" + std::to_string(maxDiff(c, g)));
}

void testGreens(Model &model){
	Solver::ChebyshevExpander cpu, gpu;
	configure(cpu, model, 256, false);
	configure(gpu, model, 256, true);
	std::vector<cplx> c = cpu.calculateCoefficients({1, 1, 0}, {1, 1, 0});

	const Type types[] = {
		Type::Advanced, Type::Retarded, Type::Principal,
		Type::NonPrincipal
	};
	const char *names[] = {
		"advanced", "retarded", "principal", "nonprincipal"
	};
	for(int t = 0; t < 4; t++){
		std::vector<cplx> a = cpu.generateGreensFunction(c, types[t]);
		std::vector<cplx> b = gpu.generateGreensFunction(c, types[t]);
		report(std::string("greens_") + names[t], sameBits(a, b),
			"max|diff|=" + std::to_string(maxDiff(a, b)));
	}

	//Changing the number of coefficients drops the device table
	//(ChebyshevExpander.h:414-420); the next call uploads a new one.
	cpu.setNumCoefficients(128);
	gpu.setNumCoefficients(128);
	std::vector<cplx> c2 = cpu.calculateCoefficients({4, 1, 1}, {4, 1, 1});
	std::vector<cplx> a = cpu.generateGreensFunction(c2, Type::Retarded);
	std::vector<cplx> b = gpu.generateGreensFunction(c2, Type::Retarded);
	report("greens_after_table_reload", sameBits(a, b),
		"max|diff|=" + std::to_string(maxDiff(a, b)));
}

void testLDOS(Model &model){
	Solver::ChebyshevExpander cpu, gpu;
	configure(cpu, model, 256, false);
	configure(gpu, model, 256, true);
	PropertyExtractor::ChebyshevExpander peCPU(cpu), peGPU(gpu);
	peCPU.setEnergyWindow(-4, 4, 301);
	peGPU.setEnergyWindow(-4, 4, 301);

	std::vector<Index> patterns = {{0, 0, 0}, {2, 3, 1}, {5, 1, IDX_ALL}};
	Property::LDOS a = peCPU.calculateLDOS(patterns);
	Property::LDOS b = peGPU.calculateLDOS(patterns);
	const std::vector<double> &da = a.getData();
	const std::vector<double> &db = b.getData();
	double d = da.size() == db.size() ? 0 : INFINITY;
	for(size_t n = 0; n < da.size() && n < db.size(); n++)
		d = std::fmax(d, std::fabs(da[n] - db[n]));
	const bool ok = da.size() == db.size() && da.size() == 4*301
		&& std::memcmp(da.data(), db.data(), da.size()*sizeof(double))
			== 0;
	report("ldos_property_extractor", ok,
		"values=" + std::to_string(db.size()) + " max|diff|="
		+ std::to_string(d));
}

// Bitwise equality of two lists of 2x2 spin matrices; d receives the
// largest entry difference.
bool sameSpinMatrices(
	const std::vector<SpinMatrix> &a, const std::vector<SpinMatrix> &b,
	double &d
){
	d = a.size() == b.size() ? 0 : INFINITY;
	bool ok = a.size() == b.size();
	for(size_t n = 0; n < a.size() && n < b.size(); n++){
		for(unsigned int r = 0; r < 2; r++){
			for(unsigned int c = 0; c < 2; c++){
				const cplx x = a[n].at(r, c), y = b[n].at(r, c);
				d = std::fmax(d, std::abs(x - y));
				ok = ok && std::memcmp(&x, &y, sizeof(cplx)) == 0;
			}
		}
	}
	return ok;
}

// TBTK's other ChebyshevExpander properties (spin-polarized LDOS, density,
// magnetization, expectation values; PropertyExtractor/ChebyshevExpander.cpp
// :297-327,584-720) call calculateCoefficients and generateGreensFunction
// once per (to, from) pair, so on the seam their recursions and energy sums
// run on the device; they must match the CPU path bit for bit.
void testProperties(Model &model){
	model.setTemperature(300);
	model.setChemicalPotential(0.1);
	Solver::ChebyshevExpander cpu, gpu;
	configure(cpu, model, 256, false);
	configure(gpu, model, 256, true);
	PropertyExtractor::ChebyshevExpander peCPU(cpu), peGPU(gpu);
	peCPU.setEnergyWindow(-4, 4, 301);
	peGPU.setEnergyWindow(-4, 4, 301);

	std::vector<Index> spinPatterns = {{2, 3, IDX_SPIN}, {0, 5, IDX_SPIN}};
	Property::SpinPolarizedLDOS sa
		= peCPU.calculateSpinPolarizedLDOS(spinPatterns);
	Property::SpinPolarizedLDOS sb
		= peGPU.calculateSpinPolarizedLDOS(spinPatterns);
	double d;
	bool ok = sameSpinMatrices(sa.getData(), sb.getData(), d)
		&& sb.getData().size() == 2*301;
	report("spin_polarized_ldos", ok,
		"values=" + std::to_string(sb.getData().size()) + " max|diff|="
		+ std::to_string(d));

	std::vector<Index> densityPatterns = {{IDX_ALL, 2, IDX_ALL}};
	Property::Density da = peCPU.calculateDensity(densityPatterns);
	Property::Density db = peGPU.calculateDensity(densityPatterns);
	const std::vector<double> &xa = da.getData(), &xb = db.getData();
	d = xa.size() == xb.size() ? 0 : INFINITY;
	for(size_t n = 0; n < xa.size() && n < xb.size(); n++)
		d = std::fmax(d, std::fabs(xa[n] - xb[n]));
	ok = xa.size() == xb.size() && xa.size() == 12
		&& std::memcmp(xa.data(), xb.data(), xa.size()*sizeof(double))
			== 0;
	report("density", ok,
		"values=" + std::to_string(xb.size()) + " max|diff|="
		+ std::to_string(d));

	std::vector<Index> magPatterns = {{1, 1, IDX_SPIN}, {4, 2, IDX_SPIN}};
	Property::Magnetization ma = peCPU.calculateMagnetization(magPatterns);
	Property::Magnetization mb = peGPU.calculateMagnetization(magPatterns);
	ok = sameSpinMatrices(ma.getData(), mb.getData(), d)
		&& mb.getData().size() == 2;
	report("magnetization", ok, "max|diff|=" + std::to_string(d));

	const cplx ea = peCPU.calculateExpectationValue({2, 3, 0}, {2, 3, 1});
	const cplx eb = peGPU.calculateExpectationValue({2, 3, 0}, {2, 3, 1});
	const cplx fa = peCPU.calculateExpectationValue({4, 4, 1}, {4, 4, 1});
	const cplx fb = peGPU.calculateExpectationValue({4, 4, 1}, {4, 4, 1});
	ok = std::memcmp(&ea, &eb, sizeof(cplx)) == 0
		&& std::memcmp(&fa, &fb, sizeof(cplx)) == 0 && fa.real() != 0;
	report("expectation_value", ok,
		"|diff|=" + std::to_string(std::abs(ea - eb) + std::abs(fa - fb)));
}

/* Named blocks of doubles: uint32 name length, name, uint64 count, data. */
class Dump{
public:
	explicit Dump(const char *path) : f(std::fopen(path, "wb")){}
	~Dump(){ if(f) std::fclose(f); }
	bool ok() const{ return f != nullptr; }
	void put(const std::string &name, const double *data, size_t count){
		const uint32_t n = name.size();
		const uint64_t c = count;
		std::fwrite(&n, sizeof(n), 1, f);
		std::fwrite(name.data(), 1, n, f);
		std::fwrite(&c, sizeof(c), 1, f);
		std::fwrite(data, sizeof(double), count, f);
	}
	void put(const std::string &name, const std::vector<double> &v){
		put(name, v.data(), v.size());
	}
	void put(const std::string &name, const std::vector<cplx> &v){
		put(name, reinterpret_cast<const double*>(v.data()), 2*v.size());
	}
	void put(const std::string &name, const std::vector<SpinMatrix> &v){
		std::vector<double> flat;
		for(const SpinMatrix &m : v)
			for(unsigned int r = 0; r < 2; r++)
				for(unsigned int c = 0; c < 2; c++){
					flat.push_back(m.at(r, c).real());
					flat.push_back(m.at(r, c).imag());
				}
		put(name, flat);
	}
private:
	std::FILE *f;
};

/* Every property of PropertyExtractor::ChebyshevExpander on the 6x6 model,
 * both the pattern-list and the pattern/ranges forms. */
int dump(bool gpu, const char *path){
	Model model;
	model.setVerbose(false);
	buildModel(model);
	model.setTemperature(300);
	model.setChemicalPotential(0.1);
	Solver::ChebyshevExpander solver;
	configure(solver, model, 256, gpu);
	PropertyExtractor::ChebyshevExpander pe(solver);
	pe.setEnergyWindow(-4, 4, 301);
	Dump out(path);
	if(!out.ok())
		return 2;
	out.put("ldos_patterns", pe.calculateLDOS({
		{0, 0, 0}, {2, 3, 1}, {5, 1, IDX_ALL}
	}).getData());
	out.put("ldos_sum", pe.calculateLDOS({{IDX_SUM_ALL, 2, IDX_ALL}}).getData());
	out.put("ldos_ranges", pe.calculateLDOS(
		{IDX_X, 3, IDX_SUM_ALL}, {6, 1, 2}
	).getData());
	out.put("greens_patterns", pe.calculateGreensFunction(
		{{{1, 1, 0}, {1, 1, IDX_ALL}}, {{2, 2, 1}, {3, 3, 1}}},
		Property::GreensFunction::Type::Retarded
	).getData());
	std::vector<Index> to = {{0, 0, 0}, {4, 1, 1}, {2, 2, 0}};
	out.put("greens_to_list", pe.calculateGreensFunctions(
		to, {2, 2, 0}, Property::GreensFunction::Type::Principal
	).getData());
	out.put("greens_advanced", pe.calculateGreensFunction(
		{3, 1, 1}, {1, 3, 0}, Property::GreensFunction::Type::Advanced
	).getData());
	out.put("density_patterns",
		pe.calculateDensity({{IDX_ALL, 2, IDX_ALL}}).getData());
	out.put("density_ranges", pe.calculateDensity(
		{IDX_X, IDX_Y, IDX_SUM_ALL}, {6, 6, 2}
	).getData());
	out.put("magnetization_patterns",
		pe.calculateMagnetization({{1, 1, IDX_SPIN}, {4, 2, IDX_SPIN}})
			.getData());
	out.put("magnetization_ranges", pe.calculateMagnetization(
		{IDX_X, 2, IDX_SPIN}, {6, 1, 2}
	).getData());
	out.put("sp_ldos_patterns",
		pe.calculateSpinPolarizedLDOS({{2, 3, IDX_SPIN}}).getData());
	out.put("sp_ldos_ranges", pe.calculateSpinPolarizedLDOS(
		{IDX_X, 0, IDX_SPIN}, {6, 1, 2}
	).getData());
	std::vector<cplx> ev = {
		pe.calculateExpectationValue({2, 3, 0}, {2, 3, 1}),
		pe.calculateExpectationValue({4, 4, 1}, {4, 4, 1})
	};
	out.put("expectation_values", ev);
	return 0;
}

/* L x L square lattice with spin, periodic, hopping -1, a Zeeman term
 * -0.5*(1 - 2s) and on-site disorder in [-1, 1] from a fixed sequence. */
void buildLattice(Model &model, int L){
	unsigned int state = 2024u;
	auto next = [&state](){
		state = state*1664525u + 1013904223u;
		return ((state >> 8) & 0xffff)/32767.5 - 1.0;
	};
	for(int x = 0; x < L; x++){
		for(int y = 0; y < L; y++){
			const double w = next();
			for(int s = 0; s < 2; s++){
				model << HoppingAmplitude(
					w - 0.5*(1 - 2*s), {x, y, s}, {x, y, s}
				);
				model << HoppingAmplitude(
					-1.0, {(x + 1)%L, y, s}, {x, y, s}
				) + HC;
				model << HoppingAmplitude(
					-1.0, {x, (y + 1)%L, s}, {x, y, s}
				) + HC;
			}
		}
	}
	model.construct();
}

int timeLDOS(){
	const int L = 256, sites = 64, M = 1024, E = 1000;
	Model model;
	model.setVerbose(false);
	buildLattice(model, L);
	Solver::ChebyshevExpander solver;
	solver.setVerbose(false);
	solver.setModel(model);
	solver.setScaleFactor(10);
	solver.setNumCoefficients(M);
	solver.setBroadening(1e-3);
	solver.setUseLookupTable(true);
	solver.setCalculateCoefficientsOnGPU(true);
	solver.setGenerateGreensFunctionsOnGPU(true);
	PropertyExtractor::ChebyshevExpander pe(solver);
	pe.setEnergyWindow(-9.9, 9.9, E);
	std::vector<Index> patterns;
	unsigned int state = 7u;
	for(int n = 0; n < sites; n++){
		state = state*1664525u + 1013904223u;
		const int site = (state >> 8) % (L*L);
		patterns.push_back({site/L, site%L, n % 2});
	}
	auto run = [&](const char *precision, double &seconds){
		setenv("TBTK_B200_PRECISION", precision, 1);
		const auto t0 = std::chrono::steady_clock::now();
		Property::LDOS ldos = pe.calculateLDOS(patterns);
		seconds = std::chrono::duration<double>(
			std::chrono::steady_clock::now() - t0
		).count();
		return ldos.getData();
	};
	double warm, fp64, mixed;
	run("fp64", warm);	//device matrix, lookup table
	std::vector<double> a = run("fp64", fp64);
	std::vector<double> b = run("mixed", mixed);
	double num = 0, den = 0;
	for(int k = 0; k < sites; k++){
		double d = 0, m = 0;
		for(int e = 0; e < E; e++){
			d = std::fmax(d, std::fabs(a[(size_t)k*E + e] - b[(size_t)k*E + e]));
			m = std::fmax(m, std::fabs(a[(size_t)k*E + e]));
		}
		num = std::fmax(num, m > 0 ? d/m : d);
		den = std::fmax(den, m);
	}
	std::printf(
		"{\"sites\": %d, \"N\": %d, \"M\": %d, \"E\": %d, "
		"\"fp64_s\": %.4f, \"mixed_s\": %.4f, \"first_call_s\": %.4f, "
		"\"mixed_rel_err\": %.3e}\n",
		sites, 2*L*L, M, E, fp64, mixed, warm, num
	);
	return 0;
}

int exitShort(){
	Model model;
	model.setVerbose(false);
	buildModel(model);
	Solver::ChebyshevExpander gpu;
	configure(gpu, model, 64, true);
	std::vector<cplx> shortCoefficients(10, cplx(1, 0));
	gpu.generateGreensFunction(shortCoefficients, Type::Retarded);
	std::printf("no exit\n");
	return 0;
}

}	//End of anonymous namespace

int main(int argc, char **argv){
	Communicator::setGlobalVerbose(false);
	//Units and constants (the occupation of density and magnetization
	//needs k_B), as a TBTK application starts.
	TBTK::Initialize();
	if(argc > 1 && std::strcmp(argv[1], "exit-short") == 0)
		return exitShort();
	if(argc > 3 && std::strcmp(argv[1], "dump") == 0)
		return dump(std::strcmp(argv[2], "gpu") == 0, argv[3]);
	if(argc > 1 && std::strcmp(argv[1], "time") == 0)
		return timeLDOS();

	Model model;
	model.setVerbose(false);
	buildModel(model);

	testDevices();
	testCoefficients(model);
	testGreens(model);
	testLDOS(model);
	testProperties(model);

	std::printf("%d failure(s)\n", failures);
	return failures == 0 ? 0 : 1;
}
