// Multi-model recursion steps on real float vectors, every lane width.
// Written by gen_steps.py.
#include "kpm_multi_real.cuh"

namespace tbtkkpm {

const MultiEntry kMultiStepsReal[] = {
    TBTKKPM_MULTI_REAL_ENTRY(1, 1, 1),
    TBTKKPM_MULTI_REAL_ENTRY(1, 1, 2),
    TBTKKPM_MULTI_REAL_ENTRY(2, 1, 1),
    TBTKKPM_MULTI_REAL_ENTRY(2, 1, 2),
    TBTKKPM_MULTI_REAL_ENTRY(1, 2, 1),
    TBTKKPM_MULTI_REAL_ENTRY(1, 2, 2),
    TBTKKPM_MULTI_REAL_ENTRY(4, 1, 1),
    TBTKKPM_MULTI_REAL_ENTRY(4, 1, 2),
    TBTKKPM_MULTI_REAL_ENTRY(1, 4, 1),
    TBTKKPM_MULTI_REAL_ENTRY(1, 4, 2),
    TBTKKPM_MULTI_REAL_ENTRY(2, 4, 1),
    TBTKKPM_MULTI_REAL_ENTRY(2, 4, 2),
    TBTKKPM_MULTI_REAL_ENTRY(8, 1, 1),
    TBTKKPM_MULTI_REAL_ENTRY(8, 1, 2),
    TBTKKPM_MULTI_REAL_ENTRY(1, 8, 1),
    TBTKKPM_MULTI_REAL_ENTRY(1, 8, 2),
    TBTKKPM_MULTI_REAL_ENTRY(4, 4, 1),
    TBTKKPM_MULTI_REAL_ENTRY(4, 4, 2),
    TBTKKPM_MULTI_REAL_ENTRY(2, 8, 1),
    TBTKKPM_MULTI_REAL_ENTRY(2, 8, 2),
    TBTKKPM_MULTI_REAL_ENTRY(8, 4, 1),
    TBTKKPM_MULTI_REAL_ENTRY(8, 4, 2),
    TBTKKPM_MULTI_REAL_ENTRY(4, 8, 1),
    TBTKKPM_MULTI_REAL_ENTRY(4, 8, 2),
    TBTKKPM_MULTI_REAL_ENTRY(16, 4, 1),
    TBTKKPM_MULTI_REAL_ENTRY(16, 4, 2),
    TBTKKPM_MULTI_REAL_ENTRY(8, 8, 1),
    TBTKKPM_MULTI_REAL_ENTRY(8, 8, 2),
};
const int kNumMultiStepsReal = sizeof(kMultiStepsReal) / sizeof(kMultiStepsReal[0]);

}  // namespace tbtkkpm
