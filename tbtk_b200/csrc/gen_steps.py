"""Writes the instantiation lists of the recursion-step kernels.

    python tbtk_b200/csrc/gen_steps.py

Each listed configuration (threads per row, complex values per thread,
register cap as min blocks per SM) is compiled into libtbtkkpm.so; the
driver's defaults and the autotuner choose among them; callers list them
through tbtkkpm_step_configs / tbtkkpm_matrix_step_configs.
"""
import pathlib

HERE = pathlib.Path(__file__).resolve().parent

SHAPES_FP64 = [(1, 1), (2, 1), (4, 1), (8, 1), (16, 1), (32, 1), (16, 2), (32, 2), (16, 4), (32, 4)]
SHAPES_MIXED = [(1, 1), (2, 1), (1, 2), (4, 1), (1, 4), (4, 2), (8, 2), (16, 2), (8, 4), (32, 2), (16, 4), (8, 8),
                (32, 4), (16, 8), (32, 8)]
MINBS = [1, 2, 3, 4]

UNITS = [
    ("steps_fp64.cu", "kStepsFP64", "kClassFP64", "double2", "Exact64", "false", SHAPES_FP64,
     "Recursion steps on complex128 vectors in the reference operation order."),
    ("steps_mixed.cu", "kStepsMixed", "kClassMixed", "float2", "Wide64", "false", SHAPES_MIXED,
     "Recursion steps on complex64 vectors with FP64 arithmetic."),
    ("steps_mixed_dots.cu", "kStepsMixedDots", "kClassMixedDots", "float2", "Wide64", "true",
     SHAPES_MIXED,
     "Recursion steps on complex64 vectors with the FP64 doubling dot products."),
]


# Bulk-copy kernels (one warp per row, a ring of S stages per warp, WPB
# warps per block): complex values per lane and (S, WPB) variants that fit
# the 227 KB of shared memory a block may use.
BULK_VPT = {"double2": [1, 2, 4], "float2": [1, 2, 4, 8]}
BULK_VARIANTS = [(2, 2), (3, 2), (2, 4), (3, 4), (4, 4), (2, 8), (3, 8)]
SMEM_LIMIT = 227 * 1024
STAGE_META = 384  # StageMeta rounded up to 128 B (kpm_bulk.cuh)
WMAX = 12


# cp.async-staged kernels (complex64 only): values per lane, stages, staged
# entries per row, warps per block.
ASYNC_VPT = [1, 2, 4]
ASYNC_STAGES = [2, 3, 4]
ASYNC_WMAX = [6, 10]
ASYNC_WPB = [4]


def async_smem(vpt, s, wmax, wpb):
    return s * wpb * (wmax + 1) * 32 * vpt * 8 + wpb * 32 * 2 * 8


def bulk_smem(V, vpt, s, wpb, dots):
    size = {"double2": 16, "float2": 8}[V]
    stage = STAGE_META + (WMAX + 1) * 32 * vpt * size
    return s * wpb * stage + (wpb * 32 * 2 * 16 if dots == "true" else 0)


# Multi-model (server) steps: lane width -> (threads per row, values per
# thread) shapes, each with the register caps MULTI_MINBS.
MULTI_SHAPES = {1: [(1, 1)], 2: [(2, 1), (1, 2)], 4: [(4, 1), (2, 2), (1, 4)], 8: [(4, 2), (2, 4), (8, 1)],
                16: [(8, 2), (4, 4), (2, 8)], 32: [(16, 2), (8, 4), (4, 8)],
                64: [(32, 2), (16, 4), (8, 8)]}
MULTI_MINBS = [1, 2]
# the same for real float vectors (values per thread are real floats)
# (16 values per thread at widths 16 and 32 spilled 240-380 bytes and lost
# to (2, 8) and (4, 8) in the server's autotuner on the uneven batch)
MULTI_REAL_SHAPES = {1: [(1, 1)], 2: [(2, 1), (1, 2)], 4: [(4, 1), (1, 4)], 8: [(2, 4), (8, 1), (1, 8)],
                     16: [(4, 4), (2, 8)], 32: [(8, 4), (4, 8)], 64: [(16, 4), (8, 8)]}


# Tile-staged multi-model steps (kpm_multi_tiled.cuh): lane width ->
# (threads per row, values per thread, rows per tile, consumer warps,
# blocks per SM).  Rows of a real width below 4 or a complex width below 2
# are under the 16 bytes a bulk copy moves at least, so those widths keep
# the register-staged steps.
# The last field is the conversion split CV of kpm_multi_tiled (0: every
# conversion an instruction of the XU pipe; 51: the first 5 gathers and
# j_{n-1} widened on the integer pipe).  The doubling terms' fixed point on
# the integer pipe too (an exact emulation of the conversion's rounding in
# integer instructions) measured 1.4-1.5x slower on the 2048^2 and 512^2
# lattices at 32 and 64 lanes and was dropped.
MULTI_TILED_REAL = {4: [(1, 4, 64, 2, 4, 0), (1, 4, 64, 2, 2, 0)],
                    8: [(2, 4, 64, 4, 2, 0), (1, 8, 64, 2, 4, 0), (2, 4, 64, 4, 2, 51)],
                    16: [(4, 4, 64, 8, 2, 0), (2, 8, 64, 4, 2, 0), (4, 4, 64, 8, 2, 51),
                         (2, 8, 64, 4, 2, 51)],
                    32: [(8, 4, 64, 16, 1, 0), (4, 8, 64, 8, 2, 0), (8, 4, 64, 16, 1, 51),
                         (4, 8, 64, 8, 2, 51)],
                    64: [(8, 8, 64, 16, 1, 0), (16, 4, 64, 16, 1, 0), (8, 8, 64, 16, 1, 51),
                         (8, 8, 64, 16, 1, 50)]}
MULTI_TILED_CPLX = {2: [(1, 2, 64, 2, 4, 0), (2, 1, 32, 2, 4, 0)],
                    4: [(2, 2, 64, 4, 2, 0), (1, 4, 64, 2, 4, 0)],
                    8: [(4, 2, 32, 4, 2, 0), (2, 4, 64, 4, 2, 0)],
                    16: [(8, 2, 32, 8, 2, 0), (4, 4, 32, 4, 2, 0), (8, 2, 32, 8, 2, 41)],
                    32: [(8, 4, 32, 8, 2, 0), (16, 2, 32, 16, 1, 0), (8, 4, 32, 8, 2, 41)],
                    64: [(16, 4, 16, 8, 2, 0), (8, 8, 32, 8, 2, 0), (16, 4, 16, 8, 2, 41)]}


def write_multi_tiled():
    lines = ["// Tile-staged multi-model recursion steps (kpm_multi_tiled.cuh).",
             "// Written by gen_steps.py.", '#include "kpm_multi_tiled.cuh"', "", "namespace tbtkkpm {", ""]
    for table, cplx, shapes in (("kMultiTiled", "true", MULTI_TILED_CPLX),
                                ("kMultiTiledReal", "false", MULTI_TILED_REAL)):
        lines.append(f"const MultiEntry {table}[] = {{")
        for w, cfgs in shapes.items():
            for (t, p, r, cw, bps, cv) in cfgs:
                assert t * p == w and cw * 32 % t == 0
                lines.append(f"    TBTKKPM_MULTI_TILED_ENTRY({cplx}, {t}, {p}, {r}, {cw}, {bps}, {cv}),")
        lines += ["};", f"const int kNum{table[1:]} = sizeof({table}) / sizeof({table}[0]);", ""]
    lines += ["}  // namespace tbtkkpm", ""]
    (HERE / "steps_multi_tiled.cu").write_text("\n".join(lines))


def write_multi():
    lines = ["// Multi-model recursion steps for every lane width the server offers.",
             "// Written by gen_steps.py.", '#include "kpm_multi.cuh"', "", "namespace tbtkkpm {", "",
             "const MultiEntry kMultiSteps[] = {"]
    for w, shapes in MULTI_SHAPES.items():
        for (t, p) in shapes:
            for mb in MULTI_MINBS:
                lines.append(f"    TBTKKPM_MULTI_ENTRY({t}, {p}, {mb}),")
    lines += ["};", "const int kNumMultiSteps = sizeof(kMultiSteps) / sizeof(kMultiSteps[0]);", "",
              "}  // namespace tbtkkpm", ""]
    (HERE / "steps_multi.cu").write_text("\n".join(lines))
    lines = ["// Multi-model recursion steps on real float vectors, every lane width.",
             "// Written by gen_steps.py.", '#include "kpm_multi_real.cuh"', "",
             "namespace tbtkkpm {", "", "const MultiEntry kMultiStepsReal[] = {"]
    for w, shapes in MULTI_REAL_SHAPES.items():
        for (t, p) in shapes:
            for mb in MULTI_MINBS:
                lines.append(f"    TBTKKPM_MULTI_REAL_ENTRY({t}, {p}, {mb}),")
    lines += ["};",
              "const int kNumMultiStepsReal = sizeof(kMultiStepsReal) / sizeof(kMultiStepsReal[0]);",
              "", "}  // namespace tbtkkpm", ""]
    (HERE / "steps_multi_real.cu").write_text("\n".join(lines))


# Real-vector steps of a real matrix at mixed precision (kpm_real.cuh):
# (threads per row, real values per thread) shapes with register caps
# REAL_MINBS, one table without and one with the doubling dot products.
SHAPES_REAL = [(1, 1), (2, 1), (1, 2), (4, 1), (1, 4), (8, 1), (1, 8), (2, 4), (16, 1), (4, 4), (32, 1), (8, 4), (4, 8),
               (16, 4), (8, 8), (4, 16), (32, 4), (16, 8), (32, 8)]
REAL_MINBS = [1, 2, 3]
# extra variants gathering G entries per round trip; 6 and 8 measured 14%
# and 76% slower than the default for (8, 8) on the 2048^2 lattice (spills)
REAL_GATHERS = []
# shape -> (register cap, OPT bits) variants of the dot-product table only
# (kpm_step_real: bit 0 bounds with the entries, bit 1 j_{n-1} at the start
# of its row, bit 3 the dot sums in shared memory).  Bits 0 and 1 are not
# compiled: for (8, 8) and (16, 4) on the 2048^2 lattice the defaults measured
# fastest or within 3%.  Bit 3 frees 2*VPT doubles of registers per thread:
# at 64 columns on the 2048^2 lattice (4, 16) went from 3.45 to 2.90 ms per
# step and (8, 8) from 3.52 to 3.28.  Shapes absent from SHAPES_REAL are
# compiled with bit 3 only.
# 16 values per thread won at every width from 16 to 256 columns; 32 values
# (128 KB of sums, one block per SM) measured 1.3-2.3x slower, caps of 1 and
# 3 at 16 values 1.4-1.9x slower (not compiled).
REAL_DOTS_OPTS = {
    (4, 8): [(2, 8)], (8, 4): [(2, 8)], (16, 4): [(2, 8)], (32, 4): [(2, 8)],
    (16, 8): [(2, 8)], (8, 8): [(2, 8), (3, 8)], (4, 16): [(2, 8)],
    (1, 16): [(2, 8)], (2, 16): [(2, 8)], (8, 16): [(2, 8)], (16, 16): [(2, 8)],
}
# Tile-staged steps (kpm_tiled.cuh): (threads per row, values per thread)
# shapes with (rows per tile, consumer warps, blocks per SM, widening split
# CV) variants.  Rows of real floats are staged with 16-byte chunks, so a
# thread holds 4 or 8 values.  On the 2048^2 lattice at 64 columns (8, 8)
# with 64-row tiles and 16 consumer warps took 1.46 ms per step, 32-row
# tiles at two blocks per SM 1.60 ms, both with every widening on the XU
# pipe (69% busy in the ncu capture); CV moves widenings to the integer pipe.
def _variants(bases, cvs):
    return [(r, cw, bps, cv) for (r, cw, bps) in bases for cv in cvs]


TILED_REAL = {
    (8, 8): _variants([(32, 8, 2), (64, 16, 1), (32, 4, 3), (16, 4, 4)], [0, 30, 50, 51]),
    (16, 4): _variants([(32, 8, 2), (64, 16, 1)], [0, 51]),
    (4, 4): _variants([(32, 8, 2), (64, 16, 1), (32, 4, 2), (64, 8, 3)], [0, 51]),
    (8, 4): _variants([(32, 8, 2), (64, 16, 1), (32, 4, 2)], [0, 51]),
    (16, 8): _variants([(32, 8, 2), (64, 16, 1), (16, 8, 2)], [0, 51]),
    (32, 4): _variants([(32, 8, 2), (64, 16, 1), (16, 8, 2)], [0, 51]),
    (32, 8): _variants([(16, 8, 2), (32, 16, 1), (16, 16, 1)], [0, 51]),
    # 4-8 sources: small blocks, several per SM
    (1, 4): _variants([(64, 2, 8), (64, 2, 6)], [0, 51]),
    (1, 8): _variants([(64, 2, 8), (64, 2, 6)], [0, 51]),
    (2, 4): _variants([(64, 4, 6), (64, 4, 4)], [0, 51]),
    (2, 8): _variants([(64, 4, 4), (64, 4, 6)], [0, 51]),
}
# CV >= 100: the row-pair form (two adjacent rows per thread group, each
# gathered row widened once for both; 16-row tiles and up).  On the 1024^2
# Rashba lattice at 128 columns its best 32 x 4 form took 2.60 ms per step
# against 2.14 ms for (16, 16, 1, CV 0), so only a few shapes stay compiled.
TILED_CPLX = {
    (32, 4): _variants([(16, 16, 1), (16, 8, 1), (8, 8, 1), (8, 8, 2)], [0, 40, 60, 90, 61])
    + _variants([(16, 8, 1)], [100, 151]),
    (16, 8): _variants([(16, 16, 1), (16, 8, 1), (8, 8, 1), (8, 8, 2)], [0, 60, 61]),
    (64, 4): _variants([(8, 8, 1), (8, 16, 1)], [0, 60]),
    (32, 8): _variants([(8, 8, 1), (8, 16, 1)], [0, 60]),
    (16, 4): _variants([(16, 8, 1), (32, 8, 1), (16, 8, 2), (16, 4, 3)], [0, 60])
    + _variants([(16, 8, 1)], [100]),
    (32, 2): _variants([(16, 8, 1), (16, 8, 2)], [0, 60]),
    (8, 4): _variants([(16, 8, 2), (32, 8, 1), (32, 8, 2)], [0, 60]) + _variants([(16, 4, 2)], [100]),
    # 64 threads per row pair, 2 values each: the pair form at the 16-warp
    # occupancy of the unpaired (32, 4) step; 2.19 ms against 2.14 ms there
    # (the unpaired 64 x 2 shape takes 2.72 ms; every merged gather widened
    # on the integer pipe, CV 190 / 191, 2.23 / 2.24 ms)
    (64, 2): _variants([(16, 16, 1)], [100, 151]),
    (8, 2): _variants([(32, 8, 2), (16, 8, 2)], [0, 60]),
    # 2-8 sources: small blocks, several per SM
    (1, 2): _variants([(64, 2, 8), (64, 2, 6)], [0, 60]),
    (1, 4): _variants([(64, 2, 8)], [0, 60]),
    (2, 2): _variants([(64, 4, 6)], [0, 60]),
    (2, 4): _variants([(64, 4, 4), (64, 4, 6)], [0, 60]),
    (4, 2): _variants([(64, 8, 4)], [0, 60]),
}


# Tile-staged FP64 steps on complex128 vectors (kpm_step_tiled with F64):
# (threads per row, complex values per thread) -> (rows per tile, consumer
# warps, blocks per SM).  Rows of 16-byte values: B = 16 / 32 / 64 / 128
# take 256 B / 512 B / 1 KB / 2 KB per row.
TILED_FP64 = {
    (1, 1): [(64, 2, 8), (64, 2, 6), (32, 1, 8), (64, 2, 4)],
    (2, 1): [(64, 4, 6), (64, 4, 4), (32, 2, 8)],
    (4, 1): [(64, 8, 4), (64, 8, 2), (32, 4, 6)],
    (8, 1): [(64, 16, 2), (32, 8, 4), (64, 8, 3)],
    (16, 1): [(32, 8, 2), (64, 16, 1)],
    (32, 1): [(32, 8, 2), (16, 8, 2), (64, 16, 1)],
    (16, 2): [(32, 8, 2), (16, 8, 2)],
    (32, 2): [(16, 16, 1), (16, 8, 1), (8, 8, 2), (8, 8, 1)],
    (16, 4): [(16, 8, 1), (8, 8, 2)],
    (32, 4): [(8, 8, 1), (8, 16, 1)],
    (16, 8): [(8, 8, 1)],
}


def tiled_fp64_lines(cls):
    return [f"    TBTKKPM_TILED_ENTRY_F64({cls}, {t}, {p}, {r}, {cw}, {bps}),"
            for (t, p), variants in TILED_FP64.items() for (r, cw, bps) in variants
            if (cw * 32) % t == 0]


def tiled_lines(cls, cplx, dots):
    shapes = TILED_CPLX if cplx else TILED_REAL
    out = []
    for (t, p), variants in shapes.items():
        for (r, cw, bps, cv) in variants:
            if (cw * 32) % t:
                continue
            c = "true" if cplx else "false"
            out.append(f"    TBTKKPM_TILED_ENTRY({cls}, {c}, {t}, {p}, {dots}, {r}, {cw}, {bps}, {cv}),")
    return out


REAL_UNITS = [
    ("steps_real.cu", "kStepsMixedReal", "kClassMixedReal", "false",
     "Recursion steps on real float vectors of a real matrix with FP64 arithmetic."),
    ("steps_real_dots.cu", "kStepsMixedRealDots", "kClassMixedRealDots", "true",
     "Recursion steps on real float vectors of a real matrix with the doubling dot products."),
]


def write_real():
    for fname, table, cls, dots, doc in REAL_UNITS:
        lines = [f"// {doc}", "// Written by gen_steps.py.", '#include "kpm_steps.cuh"', "",
                 "namespace tbtkkpm {", "", f"const StepEntry {table}[] = {{"]
        for (t, p) in SHAPES_REAL:
            for mb in REAL_MINBS:
                lines.append(f"    TBTKKPM_REAL_ENTRY({cls}, {t}, {p}, {dots}, {mb}, 0),")
            if p >= 4:
                # a whole tight-binding row per round trip at the cap of 2
                for g in REAL_GATHERS:
                    lines.append(f"    TBTKKPM_REAL_ENTRY({cls}, {t}, {p}, {dots}, 2, {g}),")
        if dots == "true":
            for (t, p), variants in REAL_DOTS_OPTS.items():
                for mb, opt in variants:
                    lines.append(f"    TBTKKPM_REAL_ENTRY_OPT({cls}, {t}, {p}, {dots}, {mb}, {opt}),")
        lines += tiled_lines(cls, False, dots)
        lines += ["};", f"const int kNum{table[1:]} = sizeof({table}) / sizeof({table}[0]);", "",
                  "}  // namespace tbtkkpm", ""]
        (HERE / fname).write_text("\n".join(lines))


def main():
    write_multi()
    write_multi_tiled()
    write_real()
    for fname, table, cls, V, AR, dots, shapes, doc in UNITS:
        lines = [f"// {doc}", "// Written by gen_steps.py: every configuration the driver and the",
                 "// autotuner can pick.", '#include "kpm_steps.cuh"', "", "namespace tbtkkpm {", "",
                 f"const StepEntry {table}[] = {{"]
        for (t, p) in shapes:
            for mb in MINBS:
                lines.append(f"    TBTKKPM_STEP_ENTRY({cls}, {V}, {AR}, {t}, {p}, {dots}, {mb}),")
        for p in BULK_VPT[V]:
            for (s, wpb) in BULK_VARIANTS:
                if bulk_smem(V, p, s, wpb, dots) <= SMEM_LIMIT:
                    lines.append(f"    TBTKKPM_BULK_ENTRY({cls}, {V}, {AR}, {p}, {dots}, {s}, {wpb}),")
        if V == "double2":
            lines += tiled_fp64_lines(cls)
        if V == "float2":
            lines += tiled_lines(cls, True, dots)
            for p in ASYNC_VPT:
                for s in ASYNC_STAGES:
                    for wmax in ASYNC_WMAX:
                        for wpb in ASYNC_WPB:
                            if async_smem(p, s, wmax, wpb) <= SMEM_LIMIT:
                                lines.append(f"    TBTKKPM_ASYNC_ENTRY({cls}, {p}, {dots}, {s}, "
                                             f"{wmax}, {wpb}),")
        lines += ["};", f"const int kNum{table[1:]} = sizeof({table}) / sizeof({table}[0]);", "",
                  "}  // namespace tbtkkpm", ""]
        (HERE / fname).write_text("\n".join(lines))


if __name__ == "__main__":
    main()
