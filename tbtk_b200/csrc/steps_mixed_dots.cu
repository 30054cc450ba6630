// Recursion steps on complex64 vectors with the doubling dot products.
// (generated list; every configuration the driver and the autotuner can pick)
#include "kpm_steps.cuh"

namespace tbtkkpm {

const StepEntry kStepsMixedDots[] = {
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 1, 1, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 1, 1, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 1, 1, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 2, 1, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 2, 1, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 2, 1, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 4, 1, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 4, 1, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 4, 1, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 4, 2, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 4, 2, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 4, 2, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 8, 2, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 8, 2, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 8, 2, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 16, 2, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 16, 2, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 16, 2, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 8, 4, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 8, 4, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 8, 4, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 32, 2, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 32, 2, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 32, 2, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 16, 4, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 16, 4, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 16, 4, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 8, 8, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 8, 8, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 8, 8, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 32, 4, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 32, 4, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 32, 4, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 16, 8, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 16, 8, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 16, 8, false, true, 4),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 32, 8, false, true, 2),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 32, 8, false, true, 3),
    TBTKKPM_STEP_ENTRY(kClassMixedDots, float2, 32, 8, false, true, 4),
};
const int kNumStepsMixedDots = sizeof(kStepsMixedDots) / sizeof(kStepsMixedDots[0]);

}  // namespace tbtkkpm
