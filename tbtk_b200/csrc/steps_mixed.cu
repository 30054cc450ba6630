// Recursion steps on complex64 vectors with FP64 arithmetic.
// (generated list; every configuration the driver and the autotuner can pick)
#include "kpm_steps.cuh"

namespace tbtkkpm {

const StepEntry kStepsMixed[] = {
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 1, 1, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 1, 1, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 1, 1, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 2, 1, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 2, 1, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 2, 1, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 4, 1, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 4, 1, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 4, 1, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 4, 2, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 4, 2, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 4, 2, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 8, 2, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 8, 2, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 8, 2, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 16, 2, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 16, 2, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 16, 2, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 8, 4, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 8, 4, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 8, 4, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 32, 2, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 32, 2, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 32, 2, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 16, 4, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 16, 4, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 16, 4, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 8, 8, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 8, 8, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 8, 8, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 32, 4, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 32, 4, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 32, 4, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 16, 8, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 16, 8, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 16, 8, false, false, 4),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 32, 8, false, false, 2),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 32, 8, false, false, 3),
    TBTKKPM_STEP_ENTRY(kClassMixed, float2, 32, 8, false, false, 4),
};
const int kNumStepsMixed = sizeof(kStepsMixed) / sizeof(kStepsMixed[0]);

}  // namespace tbtkkpm
