"""The reference's own tests of this path, compiled unchanged against the C++
shim (arcwarden_b200/shim: the reference's API on libarcb200) and run on the
GPU. Each program prints its own checks and exits non-zero on failure.

The programs are built by `make -C arcwarden_b200/shim` (part of
__graft_entry__.build()) where the reference sources are available; a test is
skipped when its program was not built.
"""
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BUILD = ROOT / "arcwarden_b200" / "shim" / "_build"
TESTS = ["test_charge_conservation", "test_poisson_sine", "test_darwin_magnetostatic", "test_fft_roundtrip",
         "test_single_particle", "test_magnetized_boris", "test_particle_load", "test_two_stream", "test_weibel",
         "test_langmuir", "test_conservation_longrun", "test_diagnostics",
         # the Yee branch (the shim's MaxwellSimulation on AW_MODEL_YEE)
         "test_yee_langmuir", "test_yee_vacuum", "test_yee_tiled", "test_yee_vs_darwin_lowfreq"]


@pytest.mark.parametrize("name", TESTS)
def test_reference_test_passes_on_the_library(torch_cuda, name):
    exe = BUILD / name
    if not exe.exists():
        pytest.skip(f"{name} not built (make -C arcwarden_b200/shim)")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])


@pytest.mark.parametrize("args", [("64", "64", "16"), ("256", "256", "64")])
def test_reference_deposit_bench_runs_on_the_library(torch_cuda, args):
    """The reference's kernel benchmark (tools/deposit_bench.cu), compiled
    unchanged on the shim: it exits 0, and its own cross-variant agreement checks
    (the shared, tiled and sorted deposits and the shared-field push against the
    global ones, tools/deposit_bench.cu:56-65, 101-175) are within 1e-5 relative
    (the library's deposits are exact, so they agree to the last bit)."""
    import re
    exe = BUILD / "deposit_bench"
    if not exe.exists():
        pytest.skip("deposit_bench not built (make -C arcwarden_b200/shim)")
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    rels = [float(m) for m in re.findall(r"correctness .*?\(rel ([0-9.eE+-]+)\)", r.stdout)]
    assert len(rels) >= 4, r.stdout
    assert max(rels) <= 1e-5, r.stdout
