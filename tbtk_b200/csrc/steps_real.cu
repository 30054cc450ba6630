// Recursion steps on real float vectors of a real matrix with FP64 arithmetic.
// Written by gen_steps.py.
#include "kpm_steps.cuh"

namespace tbtkkpm {

const StepEntry kStepsMixedReal[] = {
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 1, 1, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 1, 1, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 1, 1, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 2, 1, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 2, 1, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 2, 1, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 4, 1, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 4, 1, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 4, 1, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 8, 1, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 8, 1, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 8, 1, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 2, 4, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 2, 4, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 2, 4, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 16, 1, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 16, 1, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 16, 1, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 4, 4, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 4, 4, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 4, 4, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 32, 1, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 32, 1, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 32, 1, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 8, 4, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 8, 4, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 8, 4, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 4, 8, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 4, 8, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 4, 8, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 16, 4, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 16, 4, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 16, 4, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 8, 8, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 8, 8, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 8, 8, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 32, 4, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 32, 4, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 32, 4, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 16, 8, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 16, 8, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 16, 8, false, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 32, 8, false, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 32, 8, false, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedReal, 32, 8, false, 3, 0),
};
const int kNumStepsMixedReal = sizeof(kStepsMixedReal) / sizeof(kStepsMixedReal[0]);

}  // namespace tbtkkpm
