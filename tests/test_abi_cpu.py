"""C-ABI boundary checks that need no GPU: the library loads, exports every
entry point include/arcb200.h declares, and its ctypes signatures match."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    hdr = (ROOT / "include" / "arcb200.h").read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(aw_\w+)\s*\(", hdr, re.M)))


def test_header_declares_the_path_entry_points():
    names = declared_symbols()
    # every reference interface the boundary replaces (include/arcb200.h comments)
    for n in ("aw_ctx_create", "aw_particles_bind", "aw_load_species", "aw_deposit_rho", "aw_deposit_rho_j",
              "aw_deposit_amu", "aw_deposit_dcu", "aw_push_es", "aw_push_em", "aw_half_step_back", "aw_migrate",
              "aw_sort_tiles", "aw_solve_es", "aw_solve_darwin_el_b", "aw_solve_darwin_et", "aw_init", "aw_step",
              "aw_run", "aw_reduce_fp64"):
        assert n in names


def test_library_exports_every_declared_symbol(aw):
    lib = aw.load_library()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_header(aw):
    names = set(declared_symbols()) - {"aw_version", "aw_step_phase_name"}
    assert names == set(aw.SIGNATURES), names ^ set(aw.SIGNATURES)


def test_version_and_last_error(aw):
    assert "sm_100a" in aw.version()
    lib = aw.load_library()
    assert lib.aw_last_error(None, 0) == aw.AW_ERR_ARG


def test_null_arguments_are_rejected_without_a_gpu(aw):
    lib = aw.load_library()
    import ctypes as C
    assert lib.aw_ctx_create(None, None, 0, None, None) == aw.AW_ERR_ARG
    g = aw.Grid(0, 8, 1.0, 1.0)
    p = aw.make_params(dt=0.1)
    h = C.c_void_p()
    assert lib.aw_ctx_create(C.byref(g), C.byref(p), 0, None, C.byref(h)) == aw.AW_ERR_ARG
    assert lib.aw_ctx_create(C.byref(aw.Grid(8, 8, 1.0, 1.0)), C.byref(p), 7, None, C.byref(h)) == aw.AW_ERR_ARG
    buf = C.create_string_buffer(256)
    lib.aw_last_error(buf, 256)
    assert b"model" in buf.value
    assert lib.aw_step(None, 0) == aw.AW_ERR_ARG
    assert lib.aw_ctx_destroy(None) == aw.AW_OK


def test_struct_layouts_match_header(aw):
    import ctypes as C
    # aw_grid: 2 int32 + 2 double = 24 bytes; aw_diag: 8 doubles
    assert C.sizeof(aw.Grid) == 24
    assert C.sizeof(aw.Diag) == 64
    assert C.sizeof(aw.SourcePtrs) == 11 * 8
    assert C.sizeof(aw.FieldPtrs) == 11 * 8
    assert C.sizeof(aw.Stats) == 48
    assert C.sizeof(aw.KernelPlan) == 12


def test_product_does_not_import_the_oracle():
    """The product never imports, links or opens anything under oracle/."""
    pkg = ROOT / "arcwarden_b200"
    for f in list(pkg.rglob("*.py")) + list(pkg.rglob("*.cu")) + list(pkg.rglob("*.h")) + list(pkg.rglob("*.cuh")):
        txt = f.read_text()
        for bad in ("import oracle", "from oracle", "liboracle", "libarcref", "oracle/_", "refsim"):
            assert bad not in txt, (f, bad)


@pytest.mark.parametrize("bad", [-1])
def test_missing_library_fails_loudly(aw, tmp_path, bad):
    with pytest.raises(aw.ArcError):
        aw.load_library(tmp_path / "nope.so")
