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
    assert lib.pts_abi_version() == 3


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
    d.nout, d.precision, d.mixed_inner = 10, 1, 7
    assert lib.pts_create(ctypes.byref(d), ctypes.byref(ctx)) == _abi.PTS_E_INVAL
    assert b"mixed_inner" in lib.pts_last_error(None)
    d.precision, d.mixed_inner, d.nout = 0, 0, 0
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


def test_adjoint_and_batch_descriptions_are_validated_without_a_device():
    """The adjoint flag only exists for the 3D explicit-index FP64 two-kernel path; a batch
    needs instances of at least 3x3 cells, a positive box and a known tile shape."""
    import ptstokes
    from ptstokes import _abi
    lib = ptstokes.load()
    d = _abi.PtsDesc()
    d.nx = d.ny = d.nz = 9
    d.nout, d.lx, d.ly, d.lz = 10, 10.0, 10.0, 10.0
    ctx = ctypes.c_void_p()
    d.adjoint = 1
    for variant, precision, single_pass in ((0, 0, 0), (3, 0, 0), (5, 1, 0), (5, 0, 1), (4, 0, 2)):
        d.variant, d.precision, d.single_pass = variant, precision, single_pass
        assert lib.pts_create(ctypes.byref(d), ctypes.byref(ctx)) == _abi.PTS_E_INVAL, (variant, precision)
        assert b"adjoint" in lib.pts_last_error(None) or b"mixed" in lib.pts_last_error(None)

    bd = _abi.PtsBatchDesc()
    bd.nout, bd.tile, bd.eps = 100, 0, 1e-8
    inst = (_abi.PtsBatchInstance * 2)()
    inst[0] = _abi.PtsBatchInstance(31, 31, 10.0, 10.0, 1e-3, 1.0, 0.0, 1.0)
    inst[1] = _abi.PtsBatchInstance(2, 31, 10.0, 10.0, 1e-3, 1.0, 0.0, 1.0)
    b = ctypes.c_void_p()
    assert lib.pts_batch_create(ctypes.byref(bd), inst, 2, ctypes.byref(b)) == _abi.PTS_E_INVAL
    inst[1] = _abi.PtsBatchInstance(31, 31, -1.0, 10.0, 1e-3, 1.0, 0.0, 1.0)
    assert lib.pts_batch_create(ctypes.byref(bd), inst, 2, ctypes.byref(b)) == _abi.PTS_E_INVAL
    inst[1] = inst[0]
    bd.tile = 4
    assert lib.pts_batch_create(ctypes.byref(bd), inst, 2, ctypes.byref(b)) == _abi.PTS_E_INVAL
    bd.tile, bd.nout = 0, 0
    assert lib.pts_batch_create(ctypes.byref(bd), inst, 2, ctypes.byref(b)) == _abi.PTS_E_INVAL
    assert lib.pts_batch_create(ctypes.byref(bd), inst, 0, ctypes.byref(b)) == _abi.PTS_E_INVAL


def test_field_table_covers_the_adjoint_and_damping_fields():
    """The Python field names follow the header's pts_field enum, new fields included."""
    from ptstokes import _abi
    hdr = open(os.path.join(ROOT, "include", "ptstokes.h")).read()
    enum = hdr[hdr.index("enum pts_field"):]
    enum = enum[:enum.index("PTS_F_COUNT")]
    ids = re.findall(r"PTS_F_[A-Z_]+", enum)
    assert len(ids) == len(_abi.FIELDS)
    assert ids[-8:] == ["PTS_F_FX", "PTS_F_FY", "PTS_F_FZ", "PTS_F_GRAD", "PTS_F_DTAU_VX", "PTS_F_DTAU_VY",
                        "PTS_F_DTAU_VZ", "PTS_F_DTAU_PT"]
    assert _abi.FIELDS[-8:] == ["Fx", "Fy", "Fz", "grad", "dtVx", "dtVy", "dtVz", "dtPt"]


def test_variant_table_matches_the_header():
    """pts_variant values, the damped variants included, and their validation without a device."""
    import ptstokes
    from ptstokes import _abi
    hdr = open(os.path.join(ROOT, "include", "ptstokes.h")).read()
    enum = hdr[hdr.index("enum pts_variant"):]
    enum = re.sub(r"/\*.*?\*/", "", enum[:enum.index("};")], flags=re.S)
    vals = {m.group(1): int(m.group(2)) for m in re.finditer(r"(PTS_\w+)\s*=\s*(\d+)", enum)}
    assert vals["PTS_2D_V_DAMP"] == _abi.VARIANTS["2d_v_damp"] == 6
    assert vals["PTS_2D_VE_DAMP"] == _abi.VARIANTS["2d_ve_damp"] == 7
    assert vals["PTS_3D_V_DAMP"] == _abi.VARIANTS["3d_v_damp"] == 8
    assert sorted(vals.values()) == sorted(_abi.VARIANTS.values())
    lib = ptstokes.load()
    d = _abi.PtsDesc()
    d.nx = d.ny = d.nz = 9
    d.nout, d.lx, d.ly, d.lz = 10, 10.0, 10.0, 10.0
    ctx = ctypes.c_void_p()
    d.variant = 9
    assert lib.pts_create(ctypes.byref(d), ctypes.byref(ctx)) == _abi.PTS_E_INVAL
    for v in (7, 8):
        d.variant, d.precision, d.adjoint = v, 1, 0
        assert lib.pts_create(ctypes.byref(d), ctypes.byref(ctx)) == _abi.PTS_E_INVAL
        d.precision, d.adjoint = 0, 1
        assert lib.pts_create(ctypes.byref(d), ctypes.byref(ctx)) == _abi.PTS_E_INVAL
    d.adjoint = 0
    assert lib.pts_set_damping(None, 4.0, 2.0, 1.0, 3.0) == _abi.PTS_E_INVAL
