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
