/* The GPU functions of TBTK's Solver::ChebyshevExpander over libtbtkkpm.
 *
 * Drop-in for Lib/src/cuda/ChebyshevSolver.cu (and Lib/src/nocuda/
 * ChebyshevSolver.cpp): TBTK compiles one of those files to provide the
 * private members calculateCoefficientsGPU, generateGreensFunctionGPU,
 * loadLookupTableGPU and destroyLookupTableGPU declared in
 * Lib/include/TBTK/Solver/ChebyshevExpander.h:319-392.  Building TBTK with
 * this file instead routes them to the B200 kernels through the C ABI of
 * include/tbtkkpm.h; user code keeps selecting them with the reference's
 * setCalculateCoefficientsOnGPU / setGenerateGreensFunctionsOnGPU flags.
 *
 * Semantics kept from the reference:
 *  - the Hamiltonian is the CSR of HoppingAmplitudeSet::getSparseMatrix()
 *    (ChebyshevExpander.cpp:142-147), bit for bit; the seam keeps it on the
 *    device per (model, scale factor, device) and rebuilds it whenever the
 *    model's amplitudes differ from those it was built from, amplitude
 *    callbacks evaluated on every call as in the reference
 *    (B200::deviceMatrix, KPMSeamB200.h);
 *  - a device comes from GPUResourceManager::allocateDevice / freeDevice
 *    (ChebyshevSolver.cu:93-100,630);
 *  - the lookup table is the Solver's host table copied to every device
 *    (ChebyshevSolver.cu:672-760); generatingFunctionLookupTable_device
 *    holds one table handle per device;
 *  - failures end in TBTKExit (message on Streams::err, exit(1)).
 * Beyond the reference: all four Green's function types run on the GPU (the
 * reference's device path accepts Retarded only, ChebyshevSolver.cu:811-818).
 */
#include "TBTK/GPUResourceManager.h"
#include "TBTK/Solver/ChebyshevExpander.h"
#include "TBTK/Streams.h"
#include "TBTK/TBTKMacros.h"

#include "KPMSeamB200.h"
#include "tbtkkpm.h"

#include <complex>
#include <vector>

using namespace std;

namespace TBTK{
namespace Solver{

namespace{

/* TBTKExit expands to several statements, so it needs the braces. */
void check(int status, const char *where){
	if(status != TBTKKPM_OK){
		TBTKExit(where, tbtkkpm_last_error(), "");
	}
}

int typeCode(ChebyshevExpander::Type type){
	switch(type){
	case ChebyshevExpander::Type::Advanced:
		return TBTKKPM_ADVANCED;
	case ChebyshevExpander::Type::Retarded:
		return TBTKKPM_RETARDED;
	case ChebyshevExpander::Type::Principal:
		return TBTKKPM_PRINCIPAL;
	case ChebyshevExpander::Type::NonPrincipal:
		return TBTKKPM_NONPRINCIPAL;
	default:
		TBTKExit(
			"Solver::ChebyshevExpander::generateGreensFunctionGPU()",
			"Unknown Green's function type.",
			"This should never happen, contact the developer."
		);
	}
}

/* One device's table handles live in an array of this many entries; the
 * array is stored in generatingFunctionLookupTable_device. */
tbtkkpm_table **tables(complex<double> ***p){
	return reinterpret_cast<tbtkkpm_table**>(p);
}

}	//End of anonymous namespace

vector<complex<double>> ChebyshevExpander::calculateCoefficientsGPU(
	Index to,
	Index from
){
	vector<Index> toVector;
	toVector.push_back(to);

	return calculateCoefficientsGPU(toVector, from)[0];
}

vector<vector<complex<double>>> ChebyshevExpander::calculateCoefficientsGPU(
	vector<Index> &to,
	Index from
){
	TBTKAssert(
		scaleFactor > 0,
		"ChebyshevExpander::calculateCoefficientsGPU()",
		"Scale factor must be larger than zero.",
		"Use ChebyshevExpander::setScaleFactor() to set scale factor."
	);
	TBTKAssert(
		numCoefficients > 0,
		"ChebyshevExpander::calculateCoefficients()",
		"numCoefficients has to be larger than zero.",
		""
	);

	const HoppingAmplitudeSet &hoppingAmplitudeSet
		= getModel().getHoppingAmplitudeSet();
	const unsigned int fromBasisIndex
		= hoppingAmplitudeSet.getBasisIndex(from);
	vector<uint32_t> toBasisIndices;
	for(unsigned int n = 0; n < to.size(); n++){
		toBasisIndices.push_back(
			hoppingAmplitudeSet.getBasisIndex(to[n])
		);
	}

	GPUResourceManager &gpu = GPUResourceManager::getInstance();
	const int device = gpu.allocateDevice();
	check(
		tbtkkpm_set_device(device),
		"ChebyshevExpander::calculateCoefficientsGPU()"
	);
	std::shared_ptr<tbtkkpm_matrix> matrix = B200::deviceMatrix(
		getModel(),
		scaleFactor,
		device,
		"ChebyshevExpander::calculateCoefficientsGPU()"
	);
	vector<complex<double>> flat((size_t)to.size()*numCoefficients);
	const int status = tbtkkpm_moments(
		matrix.get(),
		fromBasisIndex,
		toBasisIndices.data(),
		toBasisIndices.size(),
		numCoefficients,
		broadening,
		reinterpret_cast<double*>(flat.data())
	);
	matrix.reset();
	gpu.freeDevice(device);
	check(status, "ChebyshevExpander::calculateCoefficientsGPU()");

	vector<vector<complex<double>>> coefficients(to.size());
	for(unsigned int n = 0; n < to.size(); n++){
		coefficients[n].assign(
			flat.begin() + (size_t)n*numCoefficients,
			flat.begin() + (size_t)(n + 1)*numCoefficients
		);
	}

	return coefficients;
}

void ChebyshevExpander::loadLookupTableGPU(){
	TBTKAssert(
		generatingFunctionLookupTable.getIsValid(),
		"ChebyshevExpander::loadLookupTableGPU()",
		"Lookup table has not been generated.",
		"Call ChebyshevExpander::generateLokupTable() to generate"
		<< " lookup table."
	);
	if(generatingFunctionLookupTable_device != nullptr)
		destroyLookupTableGPU();

	vector<complex<double>> host(
		(size_t)lookupTableNumCoefficients*lookupTableResolution
	);
	for(int n = 0; n < lookupTableNumCoefficients; n++)
		for(int e = 0; e < lookupTableResolution; e++)
			host[(size_t)n*lookupTableResolution + e]
				= generatingFunctionLookupTable[n][e];

	const int numDevices = GPUResourceManager::getInstance().getNumDevices();
	tbtkkpm_table **handles = new tbtkkpm_table*[numDevices];
	for(int n = 0; n < numDevices; n++){
		handles[n] = nullptr;
		check(
			tbtkkpm_set_device(n),
			"ChebyshevExpander::loadLookupTableGPU()"
		);
		check(
			tbtkkpm_table_upload(
				lookupTableNumCoefficients,
				lookupTableResolution,
				reinterpret_cast<const double*>(host.data()),
				&handles[n]
			),
			"ChebyshevExpander::loadLookupTableGPU()"
		);
	}
	generatingFunctionLookupTable_device
		= reinterpret_cast<complex<double>***>(handles);
}

void ChebyshevExpander::destroyLookupTableGPU(){
	TBTKAssert(
		generatingFunctionLookupTable_device != nullptr,
		"ChebyshevExpander::destroyLookupTableGPU()",
		"No lookup table loaded onto GPU.\n",
		""
	);

	tbtkkpm_table **handles = tables(generatingFunctionLookupTable_device);
	const int numDevices = GPUResourceManager::getInstance().getNumDevices();
	for(int n = 0; n < numDevices; n++)
		tbtkkpm_table_destroy(handles[n]);
	delete [] handles;
	generatingFunctionLookupTable_device = nullptr;
}

vector<complex<double>> ChebyshevExpander::generateGreensFunctionGPU(
	const vector<complex<double>> &coefficients,
	Type type
){
	ensureLookupTableIsReady();
	TBTKAssert(
		generatingFunctionLookupTable_device != nullptr,
		"ChebyshevExpander::generateGreensFunctionGPU()",
		"No lookup table loaded onto GPU.",
		""
	);
	TBTKAssert(
		(int)coefficients.size() >= lookupTableNumCoefficients,
		"ChebyshevExpander::generateGreensFunctionGPU()",
		"Expected at least " << lookupTableNumCoefficients
		<< " coefficients, got " << coefficients.size() << ".",
		""
	);

	GPUResourceManager &gpu = GPUResourceManager::getInstance();
	const int device = gpu.allocateDevice();
	vector<complex<double>> greensFunction(lookupTableResolution);
	int status = tbtkkpm_set_device(device);
	if(status == TBTKKPM_OK){
		status = tbtkkpm_greens(
			tables(generatingFunctionLookupTable_device)[device],
			reinterpret_cast<const double*>(coefficients.data()),
			1,
			typeCode(type),
			reinterpret_cast<double*>(greensFunction.data())
		);
	}
	gpu.freeDevice(device);
	check(status, "ChebyshevExpander::generateGreensFunctionGPU()");

	return greensFunction;
}

};	//End of namespace Solver
};	//End of namespace TBTK
