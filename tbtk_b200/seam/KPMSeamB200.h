/* Shared state of the B200 seam files (ChebyshevExpanderB200.cpp,
 * PropertyExtractorChebyshevExpanderB200.cpp).
 *
 * The reference rebuilds the Hamiltonian on every coefficient call:
 * HoppingAmplitudeSet::getSparseMatrix() (a host DOK -> CSC -> CSR
 * conversion, Lib/include/Core/TBTK/HoppingAmplitudeSet.h:397-424) in
 * Solver::ChebyshevExpander::calculateCoefficientsCPU/GPU
 * (Lib/src/Solver/ChebyshevExpander.cpp:142-147,
 * Lib/src/cuda/ChebyshevSolver.cu:102-130).  The seam instead keeps one
 * device matrix per (Model, scale factor, device) and checks on each use
 * that the model's amplitudes are those it was built from: one pass over
 * the HoppingAmplitudeSet hashes every amplitude with its to and from
 * indices (amplitude callbacks evaluated, as the reference evaluates them
 * per call).  A changed model, or a new model at the address of a destroyed
 * one, hashes differently and is rebuilt; the rebuild streams the
 * amplitudes as (row, column, value) triplets to the library's device
 * builder (tbtkkpm_matrix_create_triplets: device sort and duplicate fold,
 * the same CSR as getSparseMatrix bit for bit).
 *
 * Settings beyond the reference's API come from the environment:
 *   TBTK_B200_PRECISION  "fp64" (default: the reference's arithmetic, bit
 *                        for bit) or "mixed" (complex64 vectors, FP64
 *                        moments; LDOS by the doubling recursion)
 *   TBTK_B200_BATCH      sources per recursion batch (0 or unset: the
 *                        library's choice) */
#ifndef TBTK_B200_KPM_SEAM_H
#define TBTK_B200_KPM_SEAM_H

#include "TBTK/Model.h"

#include "tbtkkpm.h"

#include <cstdint>
#include <memory>

namespace TBTK{
namespace B200{

/* The device matrix of the model at this scale factor on this device (the
 * device must be current).  The cache keeps the matrices of the last few
 * (model, scale factor, device) triples; the returned reference keeps its
 * matrix alive while the caller uses it, evicted or not.  Failures end in
 * TBTKExit with `where` as the function name. */
std::shared_ptr<tbtkkpm_matrix> deviceMatrix(
	const Model &model,
	double scaleFactor,
	int device,
	const char *where
);

/* TBTKKPM_FP64 or TBTKKPM_MIXED from TBTK_B200_PRECISION. */
int precision();

/* Sources per recursion batch from TBTK_B200_BATCH (0: the library's). */
uint32_t batchWidth();

/* Ends in TBTKExit(where, tbtkkpm_last_error()) on a non-zero status. */
void check(int status, const char *where);

};	//End of namespace B200
};	//End of namespace TBTK

#endif
