// Recursion steps on real float vectors of a real matrix with the doubling dot products.
// Written by gen_steps.py.
#include "kpm_steps.cuh"

namespace tbtkkpm {

const StepEntry kStepsMixedRealDots[] = {
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 1, 1, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 1, 1, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 1, 1, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 2, 1, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 2, 1, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 2, 1, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 4, 1, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 4, 1, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 4, 1, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 8, 1, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 8, 1, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 8, 1, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 2, 4, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 2, 4, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 2, 4, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 16, 1, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 16, 1, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 16, 1, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 4, 4, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 4, 4, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 4, 4, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 32, 1, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 32, 1, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 32, 1, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 8, 4, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 8, 4, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 8, 4, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 4, 8, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 4, 8, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 4, 8, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 16, 4, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 16, 4, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 16, 4, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 8, 8, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 8, 8, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 8, 8, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 32, 4, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 32, 4, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 32, 4, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 16, 8, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 16, 8, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 16, 8, true, 3, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 32, 8, true, 1, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 32, 8, true, 2, 0),
    TBTKKPM_REAL_ENTRY(kClassMixedRealDots, 32, 8, true, 3, 0),
};
const int kNumStepsMixedRealDots = sizeof(kStepsMixedRealDots) / sizeof(kStepsMixedRealDots[0]);

}  // namespace tbtkkpm
