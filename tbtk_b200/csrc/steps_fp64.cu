// Recursion steps on complex128 vectors in the reference operation order.
// (generated list; every configuration the driver and the autotuner can pick)
#include "kpm_steps.cuh"

namespace tbtkkpm {

const StepEntry kStepsFP64[] = {
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 1, 1, true, false, 2),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 1, 1, true, false, 3),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 1, 1, true, false, 4),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 2, 1, true, false, 2),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 2, 1, true, false, 3),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 2, 1, true, false, 4),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 4, 1, true, false, 2),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 4, 1, true, false, 3),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 4, 1, true, false, 4),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 8, 1, true, false, 2),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 8, 1, true, false, 3),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 8, 1, true, false, 4),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 16, 1, true, false, 2),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 16, 1, true, false, 3),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 16, 1, true, false, 4),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 32, 1, true, false, 2),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 32, 1, true, false, 3),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 32, 1, true, false, 4),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 16, 2, true, false, 2),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 16, 2, true, false, 3),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 16, 2, true, false, 4),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 32, 2, true, false, 2),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 32, 2, true, false, 3),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 32, 2, true, false, 4),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 16, 4, true, false, 2),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 16, 4, true, false, 3),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 16, 4, true, false, 4),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 32, 4, true, false, 2),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 32, 4, true, false, 3),
    TBTKKPM_STEP_ENTRY(kClassFP64, double2, 32, 4, true, false, 4),
};
const int kNumStepsFP64 = sizeof(kStepsFP64) / sizeof(kStepsFP64[0]);

}  // namespace tbtkkpm
