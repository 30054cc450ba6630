// Tile-staged multi-model recursion steps (kpm_multi_tiled.cuh).
// Written by gen_steps.py.
#include "kpm_multi_tiled.cuh"

namespace tbtkkpm {

const MultiEntry kMultiTiled[] = {
    TBTKKPM_MULTI_TILED_ENTRY(true, 1, 2, 64, 2, 4, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 2, 1, 32, 2, 4, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 2, 2, 64, 4, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 1, 4, 64, 2, 4, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 4, 2, 32, 4, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 2, 4, 64, 4, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 8, 2, 32, 8, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 4, 4, 32, 4, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 8, 2, 32, 8, 2, 41),
    TBTKKPM_MULTI_TILED_ENTRY(true, 8, 4, 32, 8, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 16, 2, 32, 16, 1, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 8, 4, 32, 8, 2, 41),
    TBTKKPM_MULTI_TILED_ENTRY(true, 16, 4, 16, 8, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 8, 8, 32, 8, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(true, 16, 4, 16, 8, 2, 41),
};
const int kNumMultiTiled = sizeof(kMultiTiled) / sizeof(kMultiTiled[0]);

const MultiEntry kMultiTiledReal[] = {
    TBTKKPM_MULTI_TILED_ENTRY(false, 1, 4, 64, 2, 4, 0),
    TBTKKPM_MULTI_TILED_ENTRY(false, 1, 4, 64, 2, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(false, 2, 4, 64, 4, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(false, 1, 8, 64, 2, 4, 0),
    TBTKKPM_MULTI_TILED_ENTRY(false, 2, 4, 64, 4, 2, 51),
    TBTKKPM_MULTI_TILED_ENTRY(false, 4, 4, 64, 8, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(false, 2, 8, 64, 4, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(false, 4, 4, 64, 8, 2, 51),
    TBTKKPM_MULTI_TILED_ENTRY(false, 2, 8, 64, 4, 2, 51),
    TBTKKPM_MULTI_TILED_ENTRY(false, 8, 4, 64, 16, 1, 0),
    TBTKKPM_MULTI_TILED_ENTRY(false, 4, 8, 64, 8, 2, 0),
    TBTKKPM_MULTI_TILED_ENTRY(false, 8, 4, 64, 16, 1, 51),
    TBTKKPM_MULTI_TILED_ENTRY(false, 4, 8, 64, 8, 2, 51),
    TBTKKPM_MULTI_TILED_ENTRY(false, 8, 8, 64, 16, 1, 0),
    TBTKKPM_MULTI_TILED_ENTRY(false, 16, 4, 64, 16, 1, 0),
    TBTKKPM_MULTI_TILED_ENTRY(false, 8, 8, 64, 16, 1, 51),
    TBTKKPM_MULTI_TILED_ENTRY(false, 8, 8, 64, 16, 1, 50),
};
const int kNumMultiTiledReal = sizeof(kMultiTiledReal) / sizeof(kMultiTiledReal[0]);

}  // namespace tbtkkpm
