"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(pts\w*)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("pts_create", "pts_destroy", "pts_set_field", "pts_get_field", "pts_compute_P", "pts_compute_tau",
                 "pts_compute_dV", "pts_compute_V", "pts_compute_Pt_tau", "pts_compute_res", "pts_solve", "pts_run"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import ptstokes
    lib = ptstokes.load()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.pts_abi_version() == 2


def test_python_binding_covers_the_header():
    from ptstokes import _abi
    assert set(_abi.SIGNATURES) >= set(declared_symbols())


def test_struct_layouts_match_the_header():
    """ctypes mirrors of pts_desc / pts_check / pts_solve_info have the C sizes."""
    from ptstokes import _abi
    assert ctypes.sizeof(_abi.PtsDesc) == 4 * 6 + 8 * 11 + 4 * 8
    assert ctypes.sizeof(_abi.PtsCheck) == 9 * 8
    assert ctypes.sizeof(_abi.PtsSolveInfo) == 8 + 4 + 4 + 9 * 8


def test_create_rejects_bad_descriptions_without_a_device():
    """Argument validation happens before any CUDA call, so it is testable on the CPU."""
    import ptstokes
    from ptstokes import _abi
    lib = ptstokes.load()
    d = _abi.PtsDesc()
    d.variant, d.nx, d.ny, d.nz, d.nout, d.lx, d.ly, d.lz = 4, 2, 9, 9, 10, 10.0, 10.0, 10.0
    ctx = ctypes.c_void_p()
    assert lib.pts_create(ctypes.byref(d), ctypes.byref(ctx)) == _abi.PTS_E_INVAL
    assert b">= 3" in lib.pts_last_error(None)
    d.nx, d.variant = 9, 17
    assert lib.pts_create(ctypes.byref(d), ctypes.byref(ctx)) == _abi.PTS_E_INVAL
    d.variant, d.nout = 4, 0
    assert lib.pts_create(ctypes.byref(d), ctypes.byref(ctx)) == _abi.PTS_E_INVAL
    assert lib.pts_create(None, ctypes.byref(ctx)) == _abi.PTS_E_INVAL


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import ptstokes
    from ptstokes import _abi
    with pytest.raises(ptstokes.PtsError) as e:
        ptstokes.Solver("3d_ve_perf", 9, 9, 9)
    assert e.value.code == _abi.PTS_E_CUDA
