/* TBTK's PropertyExtractor::ChebyshevExpander over libtbtkkpm.
 *
 * Drop-in for Lib/src/PropertyExtractor/ChebyshevExpander.cpp: the class
 * declared in Lib/include/TBTK/PropertyExtractor/ChebyshevExpander.h with
 * every member defined here, so that a TBTK build links this file in place
 * of that one (as it links Lib/src/cuda or Lib/src/nocuda for the Solver's
 * GPU functions).
 *
 * What changes: the reference computes every property one index at a time
 * -- PropertyExtractor::calculate() calls a callback per index, and each
 * callback runs its own recursion through calculateGreensFunction
 * (ChebyshevExpander.cpp:455-505, 661-684; PropertyExtractor.h:849-894).
 * Here the callbacks only record the indices (with their memory offsets and
 * spin subindex); then the Chebyshev coefficients of all (to, from) pairs
 * of the call come from one batched recursion on the device when the
 * Solver computes coefficients on the GPU (setCalculateCoefficientsOnGPU):
 * every distinct from-index is one source of tbtkkpm_moments_batched, every
 * pair one target.  At TBTK_B200_PRECISION=fp64 (the default) each pair's
 * coefficients equal the reference's calculateCoefficients bit for bit (the
 * batched FP64 step keeps the reference's operation order per source), and
 * the Green's functions come from the Solver's own generateGreensFunction,
 * so every property is the reference's, bit for bit.  At
 * TBTK_B200_PRECISION=mixed the LDOS runs tbtkkpm_ldos_sites (complex64
 * vectors, doubling moments, FP64 energy sums, within 1e-6 of FP64) and the
 * other properties take mixed-precision coefficients.
 *
 * Without the GPU flag the coefficients come from the Solver's CPU path,
 * one call per distinct from-index with all its to-indices (the reference's
 * multi-to call, equal to single-to calls bit for bit).  Properties are
 * accumulated in the order the reference's callbacks would add them.
 */
#include "TBTK/GPUResourceManager.h"
#include "TBTK/PropertyExtractor/ChebyshevExpander.h"
#include "TBTK/Streams.h"
#include "TBTK/TBTKMacros.h"

#include "KPMSeamB200.h"
#include "tbtkkpm.h"

#include <cmath>
#include <complex>
#include <map>
#include <set>
#include <vector>

using namespace std;

namespace TBTK{
namespace PropertyExtractor{

namespace{

/* One index a calculate() loop visited: the index, the offset of its data
 * in the property and the spin subindex the loop reported. */
struct Visit{
	Index index;
	int offset;
	int spinIndex;
};

/* The visits of the calculate() loop running on this thread. */
thread_local vector<Visit> *visits = nullptr;

void record(const Index &index, int offset, int spinIndex){
	TBTKAssert(
		visits != nullptr,
		"PropertyExtractor::ChebyshevExpander",
		"A property callback ran outside a calculate() loop.",
		""
	);
	visits->push_back({index, offset, spinIndex});
}

/* Runs `loop` (a calculate() call of the base class) with the callbacks
 * recording into the returned list. */
template<typename Loop>
vector<Visit> collect(Loop loop){
	vector<Visit> list;
	vector<Visit> *outer = visits;
	visits = &list;
	loop();
	visits = outer;
	return list;
}

Solver::ChebyshevExpander::Type solverType(Property::GreensFunction::Type type){
	switch(type){
	case Property::GreensFunction::Type::Advanced:
		return Solver::ChebyshevExpander::Type::Advanced;
	case Property::GreensFunction::Type::Retarded:
		return Solver::ChebyshevExpander::Type::Retarded;
	case Property::GreensFunction::Type::Principal:
		return Solver::ChebyshevExpander::Type::Principal;
	case Property::GreensFunction::Type::NonPrincipal:
		return Solver::ChebyshevExpander::Type::NonPrincipal;
	default:
		TBTKExit(
			"PropertyExtractor::ChebyshevExpander::calculateGreensFunctions()",
			"Unknown GreensFunction type.",
			"This should never happen, contact the developer."
		);
	}
	return Solver::ChebyshevExpander::Type::NonPrincipal;
}

/* (to, from) pairs of one call and their coefficients, pairs deduplicated
 * in first-appearance order. */
class Pairs{
public:
	unsigned int add(const Index &to, const Index &from){
		pair<string, string> key(to.toString(), from.toString());
		map<pair<string, string>, unsigned int>::iterator it
			= slots.find(key);
		if(it != slots.end())
			return it->second;
		const unsigned int slot = toList.size();
		slots[key] = slot;
		toList.push_back(to);
		fromList.push_back(from);
		return slot;
	}
	unsigned int size() const{ return toList.size(); }
	const Index &to(unsigned int n) const{ return toList[n]; }
	const Index &from(unsigned int n) const{ return fromList[n]; }
private:
	vector<Index> toList, fromList;
	map<pair<string, string>, unsigned int> slots;
};

/* Coefficients of every pair: one batched device recursion (GPU flag) or
 * one CPU call per distinct from-index. */
vector<vector<complex<double>>> coefficients(
	Solver::ChebyshevExpander &solver,
	const Pairs &pairs,
	int precision,
	const char *where
){
	const unsigned int K = pairs.size();
	const int M = solver.getNumCoefficients();
	vector<vector<complex<double>>> result(K);
	if(K == 0)
		return result;
	const HoppingAmplitudeSet &set
		= solver.getModel().getHoppingAmplitudeSet();
	//Sources: the distinct from-indices in order of appearance.
	map<int, unsigned int> sourceOf;
	vector<uint32_t> sources, to(K), owner(K);
	vector<vector<unsigned int>> bySource;
	for(unsigned int n = 0; n < K; n++){
		const int f = set.getBasisIndex(pairs.from(n));
		map<int, unsigned int>::iterator it = sourceOf.find(f);
		unsigned int b;
		if(it == sourceOf.end()){
			b = sources.size();
			sourceOf[f] = b;
			sources.push_back(f);
			bySource.push_back(vector<unsigned int>());
		}
		else{
			b = it->second;
		}
		owner[n] = b;
		to[n] = set.getBasisIndex(pairs.to(n));
		bySource[b].push_back(n);
	}
	if(!solver.getCalculateCoefficientsOnGPU()){
		for(unsigned int b = 0; b < sources.size(); b++){
			vector<Index> toIndices;
			for(unsigned int n : bySource[b])
				toIndices.push_back(pairs.to(n));
			vector<vector<complex<double>>> c
				= solver.calculateCoefficients(
					toIndices,
					pairs.from(bySource[b][0])
				);
			for(unsigned int k = 0; k < bySource[b].size(); k++)
				result[bySource[b][k]] = c[k];
		}
		return result;
	}
	GPUResourceManager &gpu = GPUResourceManager::getInstance();
	const int device = gpu.allocateDevice();
	B200::check(tbtkkpm_set_device(device), where);
	shared_ptr<tbtkkpm_matrix> matrix = B200::deviceMatrix(
		solver.getModel(),
		solver.getScaleFactor(),
		device,
		where
	);
	vector<complex<double>> flat((size_t)K*M);
	const int status = tbtkkpm_moments_batched(
		matrix.get(),
		sources.data(),
		sources.size(),
		to.data(),
		owner.data(),
		K,
		M,
		solver.getBroadening(),
		precision,
		reinterpret_cast<double*>(flat.data()),
		nullptr
	);
	matrix.reset();
	gpu.freeDevice(device);
	B200::check(status, where);
	for(unsigned int n = 0; n < K; n++)
		result[n].assign(flat.begin() + (size_t)n*M, flat.begin() + (size_t)(n + 1)*M);
	return result;
}

/* Green's functions of every pair (the Solver's own energy sums). */
vector<vector<complex<double>>> greensFunctions(
	Solver::ChebyshevExpander &solver,
	const vector<vector<complex<double>>> &c,
	Property::GreensFunction::Type type
){
	const Solver::ChebyshevExpander::Type t = solverType(type);
	vector<vector<complex<double>>> g(c.size());
	//The lookup table is built lazily; build it once before the threads.
	if(!c.empty())
		g[0] = solver.generateGreensFunction(c[0], t);
	#pragma omp parallel for
	for(unsigned int n = 1; n < c.size(); n++)
		g[n] = solver.generateGreensFunction(c[n], t);
	return g;
}

/* Energies of the property's window as the Solver's lookup table holds
 * them. */
vector<double> energies(const Range &window){
	vector<double> e(window.getResolution());
	for(unsigned int n = 0; n < window.getResolution(); n++)
		e[n] = window[n];
	return e;
}

const complex<double> I(0, 1);

/* occupation(E) at every energy of the window. */
template<typename Occupation>
vector<double> occupationWeights(const Range &window, Occupation occupation){
	vector<double> w(window.getResolution());
	for(unsigned int e = 0; e < window.getResolution(); e++)
		w[e] = occupation(window[e]);
	return w;
}

};	//End of anonymous namespace

ChebyshevExpander::ChebyshevExpander(Solver::ChebyshevExpander &solver){
	const Range &window = getEnergyWindow();
	TBTKAssert(
		window.getResolution() > 0,
		"PropertyExtractor::ChebyshevExpander::ChebyshevExpander()",
		"The energy resolution has to be a positive number.",
		""
	);
	TBTKAssert(
		window[0] < window.getLast(),
		"PropertyExtractor::ChebyshevExpander::ChebyshevExpander()",
		"The energy window must be accending.",
		""
	);
	TBTKAssert(
		window[0] >= -solver.getScaleFactor(),
		"PropertyExtractor::ChebyshevExpander::ChebyshevExpander()",
		"The lower bound for the energy window has to be larger than"
		<< " -solver->getScaleFactor().",
		"Use Solver::ChebyshevExpander::setScaleFactor() to set a"
		<< " larger scale factor."
	);
	TBTKAssert(
		window.getLast() <= solver.getScaleFactor(),
		"PropertyExtractor::ChebyshevExapnder::ChebysheExpander()",
		"The upper bound for the energy window has to be smaller than"
		<< " solver->getScaleFactor().",
		"Use Solver::ChebyshevExpnader::setScaleFactor() to set a"
		<< " larger scale factor."
	);
	setSolver(solver);
	setEnergyWindow(window[0], window.getLast(), window.getResolution());
}

ChebyshevExpander::~ChebyshevExpander(){
}

void ChebyshevExpander::setEnergyWindow(
	double lowerBound,
	double upperBound,
	int energyResolution
){
	PropertyExtractor::setEnergyWindow(lowerBound, upperBound, energyResolution);
	getSolver().setEnergyWindow(Range(lowerBound, upperBound, energyResolution));
}

Property::GreensFunction ChebyshevExpander::calculateGreensFunction(
	Index to,
	Index from,
	Property::GreensFunction::Type type
){
	vector<Index> toIndices(1, to);
	return calculateGreensFunctions(toIndices, from, type);
}

Property::GreensFunction ChebyshevExpander::calculateGreensFunction(
	vector<vector<Index>> patterns,
	Property::GreensFunction::Type type
){
	const HoppingAmplitudeSet &set
		= getSolver().getModel().getHoppingAmplitudeSet();
	IndexTree memoryLayout;
	vector<pair<Index, Index>> expanded;
	for(unsigned int n = 0; n < patterns.size(); n++){
		TBTKAssert(
			patterns[n].size() == 2,
			"ChebyshevExpander::calculateGreensFunction()",
			"Invalid pattern. Each pattern entry needs to contain"
			" exactly two Indices, but '"
			<< patterns[n].size() << "' found in entry '" << n << "'.",
			""
		);
		IndexTree toTree = generateIndexTree({patterns[n][0]}, set, true, true);
		IndexTree fromTree = generateIndexTree({patterns[n][1]}, set, true, true);
		for(IndexTree::ConstIterator t = toTree.cbegin(); t != toTree.cend(); ++t){
			for(
				IndexTree::ConstIterator f = fromTree.cbegin();
				f != fromTree.cend();
				++f
			){
				memoryLayout.add({*t, *f});
				expanded.push_back(make_pair(*t, *f));
			}
		}
	}
	memoryLayout.generateLinearMap();
	Property::GreensFunction greensFunction(memoryLayout, type, getEnergyWindow());

	Pairs pairs;
	vector<unsigned int> slot(expanded.size());
	for(unsigned int n = 0; n < expanded.size(); n++)
		slot[n] = pairs.add(expanded[n].first, expanded[n].second);
	vector<vector<complex<double>>> g = greensFunctions(
		getSolver(),
		coefficients(
			getSolver(),
			pairs,
			B200::precision(),
			"PropertyExtractor::ChebyshevExpander::calculateGreensFunction()"
		),
		type
	);
	vector<complex<double>> &data = greensFunction.getDataRW();
	const unsigned int E = getEnergyWindow().getResolution();
	for(unsigned int n = 0; n < expanded.size(); n++){
		const unsigned int offset = greensFunction.getOffset(
			{expanded[n].first, expanded[n].second}
		);
		for(unsigned int e = 0; e < E; e++)
			data[offset + e] = g[slot[n]][e];
	}
	return greensFunction;
}

Property::GreensFunction ChebyshevExpander::calculateGreensFunctions(
	vector<Index> &to,
	Index from,
	Property::GreensFunction::Type type
){
	solverType(type);
	Pairs pairs;
	vector<unsigned int> slot(to.size());
	for(unsigned int n = 0; n < to.size(); n++)
		slot[n] = pairs.add(to[n], from);
	vector<vector<complex<double>>> g = greensFunctions(
		getSolver(),
		coefficients(
			getSolver(),
			pairs,
			B200::precision(),
			"PropertyExtractor::ChebyshevExpander::calculateGreensFunctions()"
		),
		type
	);
	IndexTree memoryLayout;
	for(unsigned int n = 0; n < to.size(); n++)
		memoryLayout.add({to[n], from});
	memoryLayout.generateLinearMap();
	Property::GreensFunction greensFunction(memoryLayout, type, getEnergyWindow());
	vector<complex<double>> &data = greensFunction.getDataRW();
	const unsigned int E = getEnergyWindow().getResolution();
	for(unsigned int n = 0; n < to.size(); n++){
		const unsigned int offset = greensFunction.getOffset({to[n], from});
		for(unsigned int e = 0; e < E; e++)
			data[offset + e] = g[slot[n]][e];
	}
	return greensFunction;
}

complex<double> ChebyshevExpander::calculateExpectationValue(Index to, Index from){
	Property::GreensFunction greensFunction = calculateGreensFunction(
		to,
		from,
		Property::GreensFunction::Type::NonPrincipal
	);
	const vector<complex<double>> &g = greensFunction.getData();
	const Model &model = getSolver().getModel();
	const Range &window = getEnergyWindow();
	const double dE = window[1] - window[0];
	complex<double> value = 0.;
	for(unsigned int e = 0; e < window.getResolution(); e++){
		const double weight = getThermodynamicEquilibriumOccupation(window[e], model);
		value -= weight*conj(I*g[e])*dE/M_PI;
	}
	return value;
}

/* ------------------------------------------------------------ Density */

namespace{

/* NonPrincipal Green's functions G(i, i) of the visited indices, one per
 * visit. */
vector<vector<complex<double>>> diagonalGreens(
	Solver::ChebyshevExpander &solver,
	const vector<Visit> &list,
	const char *where
){
	Pairs pairs;
	vector<unsigned int> slot(list.size());
	for(unsigned int n = 0; n < list.size(); n++)
		slot[n] = pairs.add(list[n].index, list[n].index);
	vector<vector<complex<double>>> g = greensFunctions(
		solver,
		coefficients(solver, pairs, B200::precision(), where),
		Property::GreensFunction::Type::NonPrincipal
	);
	vector<vector<complex<double>>> out(list.size());
	for(unsigned int n = 0; n < list.size(); n++)
		out[n] = g[slot[n]];
	return out;
}

/* NonPrincipal Green's functions of the four spin pairs (up-up, up-down,
 * down-up, down-down) of each visited index: [visit][pair]. */
vector<vector<vector<complex<double>>>> spinGreens(
	Solver::ChebyshevExpander &solver,
	const vector<Visit> &list,
	const char *where
){
	Pairs pairs;
	vector<unsigned int> slot(4*list.size());
	for(unsigned int n = 0; n < list.size(); n++){
		for(int s = 0; s < 4; s++){
			Index to(list[n].index), from(list[n].index);
			to.at(list[n].spinIndex) = s/2;
			from.at(list[n].spinIndex) = s%2;
			slot[4*n + s] = pairs.add(to, from);
		}
	}
	vector<vector<complex<double>>> g = greensFunctions(
		solver,
		coefficients(solver, pairs, B200::precision(), where),
		Property::GreensFunction::Type::NonPrincipal
	);
	vector<vector<vector<complex<double>>>> out(list.size());
	for(unsigned int n = 0; n < list.size(); n++)
		for(int s = 0; s < 4; s++)
			out[n].push_back(g[slot[4*n + s]]);
	return out;
}

/* weight[e]: the thermodynamic equilibrium occupation at energy e of the
 * window (PropertyExtractor::getThermodynamicEquilibriumOccupation). */
void addDensity(
	Solver::ChebyshevExpander &solver,
	const Range &window,
	const vector<double> &weight,
	const vector<Visit> &list,
	vector<double> &data
){
	vector<vector<complex<double>>> g = diagonalGreens(
		solver,
		list,
		"PropertyExtractor::ChebyshevExpander::calculateDensity()"
	);
	const double dE = window[1] - window[0];
	for(unsigned int n = 0; n < list.size(); n++)
		for(unsigned int e = 0; e < window.getResolution(); e++)
			data[list[n].offset] += weight[e]*imag(g[n][e])/M_PI*dE;
}

void addMagnetization(
	Solver::ChebyshevExpander &solver,
	const Range &window,
	const vector<double> &weight,
	const vector<Visit> &list,
	vector<SpinMatrix> &data
){
	vector<vector<vector<complex<double>>>> g = spinGreens(
		solver,
		list,
		"PropertyExtractor::ChebyshevExpander::calculateMagnetization()"
	);
	const double dE = window[1] - window[0];
	for(unsigned int n = 0; n < list.size(); n++)
		for(int s = 0; s < 4; s++)
			for(unsigned int e = 0; e < window.getResolution(); e++)
				data[list[n].offset].at(s/2, s%2)
					+= weight[e]*(-I)*g[n][s][e]/M_PI*dE;
}

void addSpinPolarizedLDOS(
	Solver::ChebyshevExpander &solver,
	const Range &window,
	const vector<Visit> &list,
	vector<SpinMatrix> &data
){
	vector<vector<vector<complex<double>>>> g = spinGreens(
		solver,
		list,
		"PropertyExtractor::ChebyshevExpander::calculateSpinPolarizedLDOS()"
	);
	for(unsigned int n = 0; n < list.size(); n++)
		for(int s = 0; s < 4; s++)
			for(unsigned int e = 0; e < window.getResolution(); e++)
				data[list[n].offset + e].at(s/2, s%2) += -I*g[n][s][e]/M_PI;
}

/* LDOS of the visited indices.  FP64 and the CPU path: Im G_NP / pi from
 * the Solver's Green's functions, added in visit order.  Mixed precision on
 * the GPU: tbtkkpm_ldos_sites on the distinct basis indices (doubling
 * recursion, FP64 head, device lookup table of the window). */
void addLDOS(
	Solver::ChebyshevExpander &solver,
	const Range &window,
	const vector<Visit> &list,
	vector<double> &data
){
	const char *where = "PropertyExtractor::ChebyshevExpander::calculateLDOS()";
	const unsigned int E = window.getResolution();
	if(
		B200::precision() == TBTKKPM_MIXED
		&& solver.getCalculateCoefficientsOnGPU()
		&& !list.empty()
	){
		const HoppingAmplitudeSet &set
			= solver.getModel().getHoppingAmplitudeSet();
		map<int, unsigned int> slotOf;
		vector<uint32_t> sites;
		vector<unsigned int> slot(list.size());
		for(unsigned int n = 0; n < list.size(); n++){
			const int b = set.getBasisIndex(list[n].index);
			map<int, unsigned int>::iterator it = slotOf.find(b);
			if(it == slotOf.end()){
				slotOf[b] = sites.size();
				slot[n] = sites.size();
				sites.push_back(b);
			}
			else{
				slot[n] = it->second;
			}
		}
		GPUResourceManager &gpu = GPUResourceManager::getInstance();
		const int device = gpu.allocateDevice();
		B200::check(tbtkkpm_set_device(device), where);
		shared_ptr<tbtkkpm_matrix> matrix = B200::deviceMatrix(
			solver.getModel(),
			solver.getScaleFactor(),
			device,
			where
		);
		const vector<double> en = energies(window);
		tbtkkpm_table *table = nullptr;
		int status = tbtkkpm_table_create(
			solver.getNumCoefficients(),
			en.data(),
			E,
			solver.getScaleFactor(),
			&table
		);
		vector<double> ldos((size_t)sites.size()*E);
		if(status == TBTKKPM_OK){
			status = tbtkkpm_ldos_sites(
				matrix.get(),
				table,
				sites.data(),
				sites.size(),
				solver.getBroadening(),
				TBTKKPM_MIXED,
				ldos.data(),
				nullptr
			);
		}
		tbtkkpm_table_destroy(table);
		matrix.reset();
		gpu.freeDevice(device);
		B200::check(status, where);
		for(unsigned int n = 0; n < list.size(); n++)
			for(unsigned int e = 0; e < E; e++)
				data[list[n].offset + e] += ldos[(size_t)slot[n]*E + e];
		return;
	}
	vector<vector<complex<double>>> g = diagonalGreens(solver, list, where);
	for(unsigned int n = 0; n < list.size(); n++)
		for(unsigned int e = 0; e < E; e++)
			data[list[n].offset + e] += imag(g[n][e])/M_PI;
}

};	//End of anonymous namespace

Property::Density ChebyshevExpander::calculateDensity(Index pattern, Index ranges){
	ensureCompliantRanges(pattern, ranges);
	Property::Density density(getLoopRanges(pattern, ranges));
	Information information;
	vector<Visit> list = collect([&](){
		calculate(calculateDensityCallback, density, pattern, ranges, 0, 1, information);
	});
	addDensity(getSolver(), getEnergyWindow(), occupationWeights(getEnergyWindow(), [&](double E){
		return getThermodynamicEquilibriumOccupation(E, getSolver().getModel());
	}), list, density.getDataRW());
	return density;
}

Property::Density ChebyshevExpander::calculateDensity(vector<Index> patterns){
	const HoppingAmplitudeSet &set
		= getSolver().getModel().getHoppingAmplitudeSet();
	IndexTree allIndices = generateIndexTree(patterns, set, false, false);
	IndexTree memoryLayout = generateIndexTree(patterns, set, true, true);
	Property::Density density(memoryLayout);
	Information information;
	vector<Visit> list = collect([&](){
		calculate(calculateDensityCallback, allIndices, memoryLayout, density, information);
	});
	addDensity(getSolver(), getEnergyWindow(), occupationWeights(getEnergyWindow(), [&](double E){
		return getThermodynamicEquilibriumOccupation(E, getSolver().getModel());
	}), list, density.getDataRW());
	return density;
}

/* The position of the pattern's spin subindex (IDX_SPIN), which is fixed
 * to 0 with range 1 for the loop; no spin subindex ends in TBTKExit. */
static int takeSpinIndex(Index &pattern, Index &ranges, const char *where){
	for(unsigned int n = 0; n < pattern.getSize(); n++){
		if(pattern.at(n).isSpinIndex()){
			pattern.at(n) = 0;
			ranges.at(n) = 1;
			return n;
		}
	}
	TBTKExit(
		where,
		"No spin index indicated.",
		"Use IDX_SPIN to indicate the position of the spin index."
	);
	return -1;
}

Property::Magnetization ChebyshevExpander::calculateMagnetization(
	Index pattern,
	Index ranges
){
	Information information;
	information.setSpinIndex(takeSpinIndex(
		pattern,
		ranges,
		"PropertyExtractor::ChebyshevExpander::calculateMagnetization()"
	));
	ensureCompliantRanges(pattern, ranges);
	Property::Magnetization magnetization(getLoopRanges(pattern, ranges));
	vector<Visit> list = collect([&](){
		calculate(calculateMAGCallback, magnetization, pattern, ranges, 0, 1, information);
	});
	addMagnetization(getSolver(), getEnergyWindow(), occupationWeights(getEnergyWindow(), [&](double E){
		return getThermodynamicEquilibriumOccupation(E, getSolver().getModel());
	}), list, magnetization.getDataRW());
	return magnetization;
}

Property::Magnetization ChebyshevExpander::calculateMagnetization(
	vector<Index> patterns
){
	const HoppingAmplitudeSet &set
		= getSolver().getModel().getHoppingAmplitudeSet();
	IndexTree allIndices = generateIndexTree(patterns, set, false, true);
	IndexTree memoryLayout = generateIndexTree(patterns, set, true, true);
	Property::Magnetization magnetization(memoryLayout);
	Information information;
	vector<Visit> list = collect([&](){
		calculate(
			calculateMAGCallback,
			allIndices,
			memoryLayout,
			magnetization,
			information
		);
	});
	addMagnetization(getSolver(), getEnergyWindow(), occupationWeights(getEnergyWindow(), [&](double E){
		return getThermodynamicEquilibriumOccupation(E, getSolver().getModel());
	}), list, magnetization.getDataRW());
	return magnetization;
}

Property::LDOS ChebyshevExpander::calculateLDOS(Index pattern, Index ranges){
	ensureCompliantRanges(pattern, ranges);
	Property::LDOS ldos(getLoopRanges(pattern, ranges), getEnergyWindow());
	Information information;
	vector<Visit> list = collect([&](){
		calculate(
			calculateLDOSCallback,
			ldos,
			pattern,
			ranges,
			0,
			getEnergyWindow().getResolution(),
			information
		);
	});
	addLDOS(getSolver(), getEnergyWindow(), list, ldos.getDataRW());
	return ldos;
}

Property::LDOS ChebyshevExpander::calculateLDOS(vector<Index> patterns){
	const HoppingAmplitudeSet &set
		= getSolver().getModel().getHoppingAmplitudeSet();
	IndexTree allIndices = generateIndexTree(patterns, set, false, true);
	IndexTree memoryLayout = generateIndexTree(patterns, set, true, true);
	Property::LDOS ldos(memoryLayout, getEnergyWindow());
	Information information;
	vector<Visit> list = collect([&](){
		calculate(calculateLDOSCallback, allIndices, memoryLayout, ldos, information);
	});
	addLDOS(getSolver(), getEnergyWindow(), list, ldos.getDataRW());
	return ldos;
}

Property::SpinPolarizedLDOS ChebyshevExpander::calculateSpinPolarizedLDOS(
	Index pattern,
	Index ranges
){
	Information information;
	information.setSpinIndex(takeSpinIndex(
		pattern,
		ranges,
		"PropertyExtractor::ChebsyhevExpander::calculateSpinPolarizedLDOS()"
	));
	ensureCompliantRanges(pattern, ranges);
	Property::SpinPolarizedLDOS spinPolarizedLDOS(
		getLoopRanges(pattern, ranges),
		getEnergyWindow()
	);
	vector<Visit> list = collect([&](){
		calculate(
			calculateSP_LDOSCallback,
			spinPolarizedLDOS,
			pattern,
			ranges,
			0,
			getEnergyWindow().getResolution(),
			information
		);
	});
	addSpinPolarizedLDOS(
		getSolver(),
		getEnergyWindow(),
		list,
		spinPolarizedLDOS.getDataRW()
	);
	return spinPolarizedLDOS;
}

Property::SpinPolarizedLDOS ChebyshevExpander::calculateSpinPolarizedLDOS(
	vector<Index> patterns
){
	const HoppingAmplitudeSet &set
		= getSolver().getModel().getHoppingAmplitudeSet();
	IndexTree allIndices = generateIndexTree(patterns, set, false, true);
	IndexTree memoryLayout = generateIndexTree(patterns, set, true, true);
	Property::SpinPolarizedLDOS spinPolarizedLDOS(memoryLayout, getEnergyWindow());
	Information information;
	vector<Visit> list = collect([&](){
		calculate(
			calculateSP_LDOSCallback,
			allIndices,
			memoryLayout,
			spinPolarizedLDOS,
			information
		);
	});
	addSpinPolarizedLDOS(
		getSolver(),
		getEnergyWindow(),
		list,
		spinPolarizedLDOS.getDataRW()
	);
	return spinPolarizedLDOS;
}

/* The callbacks of the calculate() loops record the visited index; the
 * property is computed for all of them once the loop is done. */
void ChebyshevExpander::calculateDensityCallback(
	PropertyExtractor *cb_this,
	Property::Property &property,
	const Index &index,
	int offset,
	Information &information
){
	record(index, offset, information.getSpinIndex());
}

void ChebyshevExpander::calculateMAGCallback(
	PropertyExtractor *cb_this,
	Property::Property &property,
	const Index &index,
	int offset,
	Information &information
){
	record(index, offset, information.getSpinIndex());
}

void ChebyshevExpander::calculateLDOSCallback(
	PropertyExtractor *cb_this,
	Property::Property &property,
	const Index &index,
	int offset,
	Information &information
){
	record(index, offset, information.getSpinIndex());
}

void ChebyshevExpander::calculateSP_LDOSCallback(
	PropertyExtractor *cb_this,
	Property::Property &property,
	const Index &index,
	int offset,
	Information &information
){
	record(index, offset, information.getSpinIndex());
}

};	//End of namespace PropertyExtractor
};	//End of namespace TBTK
