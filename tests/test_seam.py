"""TBTK's own ChebyshevExpander classes on the B200 seam.

tests/cpp/_build/test_seam is the reference's Solver and PropertyExtractor
(compiled from its sources) linked with tbtk_b200/seam instead of
Lib/src/cuda/ChebyshevSolver.cu; it is built next to the reference sources
(tests/cpp/Makefile) and runs anywhere libtbtkkpm.so does.
"""
import os
import subprocess

import pytest

import tbtk_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(tbtk_b200.__file__)))
BINARY = os.path.join(ROOT, "tests", "cpp", "_build", "test_seam")

needs_binary = pytest.mark.skipif(
    not os.path.exists(BINARY),
    reason="seam test binary not built (needs the reference sources)")


def run(*args):
    return subprocess.run([BINARY, *args], capture_output=True, text=True,
                          timeout=600)


def has_gpu():
    import torch
    return torch.cuda.is_available()


@needs_binary
def test_seam_without_devices_exits_like_tbtk():
    """No device: GPUResourceManager's table is empty and allocateDevice
    ends the program the reference's way
    (Lib/src/Utilities/GPUResourceManager.cpp:44-50)."""
    if has_gpu():
        pytest.skip("a GPU is visible")
    r = run()
    assert r.returncode == 1
    assert "[FAIL] device_table devices=0" in r.stdout
    assert "No GPU devices available" in r.stdout + r.stderr


@pytest.mark.gpu
@needs_binary
def test_seam_matches_tbtk_cpu_path():
    if not has_gpu():
        pytest.skip("no GPU visible")
    r = run()
    lines = [l for l in r.stdout.splitlines() if l.startswith("[")]
    assert r.returncode == 0, r.stdout + r.stderr
    names = {l.split()[1] for l in lines}
    assert names == {
        "device_table", "coefficients_many_to", "coefficients_single",
        "greens_advanced", "greens_retarded", "greens_principal",
        "greens_nonprincipal", "greens_after_table_reload",
        "ldos_property_extractor", "spin_polarized_ldos", "density",
        "magnetization", "expectation_value"}
    assert all(l.startswith("[PASS]") for l in lines), r.stdout


@pytest.mark.gpu
@needs_binary
def test_seam_error_ends_in_tbtk_exit():
    r = run("exit-short")
    out = r.stdout + r.stderr
    assert r.returncode == 1, out
    assert "generateGreensFunctionGPU" in out
    assert "Expected at least 64 coefficients, got 10" in out
    assert "no exit" not in out


# ---------------------------------------------------------------------------
# The seam's PropertyExtractor::ChebyshevExpander (batched over the indices
# of a call) in place of the reference's, in tests/cpp/_build/test_pe_seam.

PE_BINARY = os.path.join(ROOT, "tests", "cpp", "_build", "test_pe_seam")

needs_pe_binary = pytest.mark.skipif(
    not os.path.exists(PE_BINARY) or not os.path.exists(BINARY),
    reason="seam test binaries not built (need the reference sources)")


def read_dump(path):
    """Named blocks of doubles written by `test_seam dump`."""
    import struct

    import numpy as np
    out = {}
    with open(path, "rb") as f:
        raw = f.read()
    pos = 0
    while pos < len(raw):
        (n,) = struct.unpack_from("<I", raw, pos)
        pos += 4
        name = raw[pos:pos + n].decode()
        pos += n
        (c,) = struct.unpack_from("<Q", raw, pos)
        pos += 8
        out[name] = np.frombuffer(raw, dtype=np.float64, count=c, offset=pos)
        pos += 8 * c
    return out


DUMP_BLOCKS = {"ldos_patterns", "ldos_sum", "ldos_ranges", "greens_patterns", "greens_to_list",
               "greens_advanced", "density_patterns", "density_ranges", "magnetization_patterns",
               "magnetization_ranges", "sp_ldos_patterns", "sp_ldos_ranges",
               "expectation_values"}


@needs_pe_binary
def test_pe_seam_cpu_path_equals_reference(tmp_path):
    """Without the GPU flags the seam's PropertyExtractor takes the Solver's
    CPU coefficients once per distinct from-index and accumulates every
    property in the reference's order: byte for byte the reference's
    output, for every property and both pattern forms."""
    ref, ours = tmp_path / "ref.bin", tmp_path / "ours.bin"
    a = subprocess.run([BINARY, "dump", "cpu", str(ref)], capture_output=True, text=True)
    b = subprocess.run([PE_BINARY, "dump", "cpu", str(ours)], capture_output=True, text=True)
    assert a.returncode == 0 and b.returncode == 0, a.stderr + b.stderr
    da, db = read_dump(ref), read_dump(ours)
    assert set(da) == DUMP_BLOCKS == set(db)
    assert ref.read_bytes() == ours.read_bytes()


@pytest.mark.gpu
@needs_pe_binary
def test_pe_seam_batched_gpu_path_equals_reference(tmp_path):
    """With the GPU flags every property's coefficients come from one
    batched device recursion per call: at FP64 byte for byte the reference
    PropertyExtractor on the CPU path; at mixed precision (complex64
    vectors, doubling LDOS) the LDOS within 1e-6 and the other properties
    within 1e-5 of it (max|x - ref| / max|ref| per block).  The checks of
    test_seam pass with the seam's PropertyExtractor too."""
    import numpy as np
    if not has_gpu():
        pytest.skip("no GPU visible")
    ref, fp64, mixed = tmp_path / "ref.bin", tmp_path / "fp64.bin", tmp_path / "mixed.bin"
    assert subprocess.run([BINARY, "dump", "cpu", str(ref)]).returncode == 0
    env = dict(os.environ, TBTK_B200_PRECISION="fp64")
    r = subprocess.run([PE_BINARY, "dump", "gpu", str(fp64)], env=env, capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert ref.read_bytes() == fp64.read_bytes()
    env["TBTK_B200_PRECISION"] = "mixed"
    r = subprocess.run([PE_BINARY, "dump", "gpu", str(mixed)], env=env, capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    da, dm = read_dump(ref), read_dump(mixed)
    for name in DUMP_BLOCKS:
        err = float(np.abs(dm[name] - da[name]).max() / np.abs(da[name]).max())
        assert err <= (1e-6 if name.startswith("ldos") else 1e-5), (name, err)
    r = subprocess.run([PE_BINARY], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
@needs_pe_binary
def test_pe_seam_ldos_of_64_sites_in_one_batch():
    """calculateLDOS of 64 sites of a 256x256 lattice with spin through
    TBTK's API: the reference's PropertyExtractor runs 64 recursions one
    after another (each on the seam's cached device matrix), the seam's runs
    them as one batch; the mixed precision stays within 1e-6 of FP64."""
    import json
    if not has_gpu():
        pytest.skip("no GPU visible")
    per_site = json.loads(run("time").stdout.strip().splitlines()[-1])
    r = subprocess.run([PE_BINARY, "time"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    batched = json.loads(r.stdout.strip().splitlines()[-1])
    print("reference PropertyExtractor:", per_site)
    print("seam PropertyExtractor:", batched)
    assert batched["mixed_rel_err"] <= 1e-6
    assert batched["fp64_s"] < per_site["fp64_s"]
