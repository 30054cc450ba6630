// Multi-model recursion steps for every lane width the server offers.
// Written by gen_steps.py.
#include "kpm_multi.cuh"

namespace tbtkkpm {

const MultiEntry kMultiSteps[] = {
    TBTKKPM_MULTI_ENTRY(1, 1, 1),
    TBTKKPM_MULTI_ENTRY(1, 1, 2),
    TBTKKPM_MULTI_ENTRY(2, 1, 1),
    TBTKKPM_MULTI_ENTRY(2, 1, 2),
    TBTKKPM_MULTI_ENTRY(1, 2, 1),
    TBTKKPM_MULTI_ENTRY(1, 2, 2),
    TBTKKPM_MULTI_ENTRY(4, 1, 1),
    TBTKKPM_MULTI_ENTRY(4, 1, 2),
    TBTKKPM_MULTI_ENTRY(2, 2, 1),
    TBTKKPM_MULTI_ENTRY(2, 2, 2),
    TBTKKPM_MULTI_ENTRY(1, 4, 1),
    TBTKKPM_MULTI_ENTRY(1, 4, 2),
    TBTKKPM_MULTI_ENTRY(4, 2, 1),
    TBTKKPM_MULTI_ENTRY(4, 2, 2),
    TBTKKPM_MULTI_ENTRY(2, 4, 1),
    TBTKKPM_MULTI_ENTRY(2, 4, 2),
    TBTKKPM_MULTI_ENTRY(8, 1, 1),
    TBTKKPM_MULTI_ENTRY(8, 1, 2),
    TBTKKPM_MULTI_ENTRY(8, 2, 1),
    TBTKKPM_MULTI_ENTRY(8, 2, 2),
    TBTKKPM_MULTI_ENTRY(4, 4, 1),
    TBTKKPM_MULTI_ENTRY(4, 4, 2),
    TBTKKPM_MULTI_ENTRY(2, 8, 1),
    TBTKKPM_MULTI_ENTRY(2, 8, 2),
    TBTKKPM_MULTI_ENTRY(16, 2, 1),
    TBTKKPM_MULTI_ENTRY(16, 2, 2),
    TBTKKPM_MULTI_ENTRY(8, 4, 1),
    TBTKKPM_MULTI_ENTRY(8, 4, 2),
    TBTKKPM_MULTI_ENTRY(4, 8, 1),
    TBTKKPM_MULTI_ENTRY(4, 8, 2),
    TBTKKPM_MULTI_ENTRY(32, 2, 1),
    TBTKKPM_MULTI_ENTRY(32, 2, 2),
    TBTKKPM_MULTI_ENTRY(16, 4, 1),
    TBTKKPM_MULTI_ENTRY(16, 4, 2),
    TBTKKPM_MULTI_ENTRY(8, 8, 1),
    TBTKKPM_MULTI_ENTRY(8, 8, 2),
};
const int kNumMultiSteps = sizeof(kMultiSteps) / sizeof(kMultiSteps[0]);

}  // namespace tbtkkpm
