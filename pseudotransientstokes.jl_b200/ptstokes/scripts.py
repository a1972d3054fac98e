"""The reference scripts' solver functions, on the GPU.

Each function mirrors the ``Stokes2D_()`` / ``Stokes3D_()`` function of one script of
PTsolvers/PseudoTransientStokes.jl and returns what it returns with USE_RETURN=true:
``(xc, yc, Pt)`` in 2D and ``(xc, yc, zc, Pt)`` in 3D. Grid sizes default to the
scripts' NX/NY/NZ environment variables (``haskey(ENV, "NX") ? parse(Int, ENV["NX"]) : ...``).

    Stokes2D            scripts/Stokes2D.jl
    Stokes2D_ve         scripts/Stokes2D_ve.jl
    Stokes2D_ve_perf    scripts/Stokes2D_ve_perf.jl
    Stokes3D_ve         scripts/stokes_3D/Stokes3D_ve_multixpu.jl (one rank)
    Stokes3D_ve_perf    scripts/stokes_3D/Stokes3D_ve_perf.jl
    Stokes3D_v          3D viscous (no reference script)
    Stokes2D0           scripts/previous_damp/Stokes2D0.jl    (damped scheme)
    Stokes2D_ve0        scripts/previous_damp/Stokes2D_ve0.jl (damped scheme)
    Stokes3D0           scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl (one rank, damped scheme)
"""
import os
import time

from . import output
from .solver import Solver


def _env(name, default):
    v = os.environ.get(name)
    return int(v) if v is not None else default


def _flag(name):
    """`haskey(ENV, name) ? parse(Bool, ENV[name]) : false` of the scripts' headers."""
    return os.environ.get(name, "false").strip().lower() in ("true", "1")


def _script(variant, nx, ny, nz, return_solver, verbose, do_save=None, do_save_viz=None, **kw):
    s = Solver(variant, nx, ny, nz, **kw)
    s.setup_inclusion(musi=kw.get("musi", 1e-3))
    t0 = time.perf_counter()
    res = s.run()
    s.sync()
    wall = time.perf_counter() - t0
    res["wall_s"] = wall
    if verbose:
        print(f"Total iters = {res['ittot']} ({len(res['iters'])} steps), time = {wall:1.3e} sec")
    if _flag("DO_SAVE") if do_save is None else do_save:  # the scripts' output/out_*.txt line
        output.save_line(s, res, wall, os.environ.get("PTS_OUTPUT_DIR", "output"))
    if _flag("DO_SAVE_VIZ") if do_save_viz is None else do_save_viz:  # the scripts' out_visu/*.mat dump
        if variant in output.MAT_FILES:
            output.save_visu(s, os.environ.get("PTS_VISU_DIR", "out_visu"))
    out = (*s.centres(), s.get("Pt"))
    if return_solver:
        return out, s, res
    s.close()
    return out


def Stokes2D(nx=None, ny=None, return_solver=False, verbose=False, **kw):
    """scripts/Stokes2D.jl:72-169 (2D viscous, pure shear, weak inclusion)."""
    return _script("2d_v", nx or _env("NX", 255), ny or _env("NY", 255), None, return_solver, verbose, **kw)


def Stokes2D_ve(nx=None, ny=None, return_solver=False, verbose=False, **kw):
    """scripts/Stokes2D_ve.jl:87-206 (2D Maxwell visco-elastic, 5 physical steps)."""
    return _script("2d_ve", nx or _env("NX", 255), ny or _env("NY", 255), None, return_solver, verbose, **kw)


def Stokes2D_ve_perf(nx=None, ny=None, return_solver=False, verbose=False, **kw):
    """scripts/Stokes2D_ve_perf.jl:80-197 (2D VE, 101 PT iterations)."""
    return _script("2d_ve_perf", nx or _env("NX", 255), ny or _env("NY", 255), None, return_solver, verbose, **kw)


def Stokes3D_ve(nx=None, ny=None, nz=None, return_solver=False, verbose=False, **kw):
    """scripts/stokes_3D/Stokes3D_ve_multixpu.jl:118-295 on one rank (5 physical steps)."""
    return _script("3d_ve", nx or _env("NX", 63), ny or _env("NY", 63), nz or _env("NZ", 63), return_solver,
                   verbose, **kw)


def Stokes3D_ve_perf(nx=None, ny=None, nz=None, return_solver=False, verbose=False, **kw):
    """scripts/stokes_3D/Stokes3D_ve_perf.jl:116-255 (201 PT iterations)."""
    return _script("3d_ve_perf", nx or _env("NX", 63), ny or _env("NY", 63), nz or _env("NZ", 63), return_solver,
                   verbose, **kw)


def Stokes3D_v(nx=None, ny=None, nz=None, return_solver=False, verbose=False, **kw):
    """3D viscous Stokes (the 3D kernels without elastic terms; no reference script)."""
    return _script("3d_v", nx or _env("NX", 63), ny or _env("NY", 63), nz or _env("NZ", 63), return_solver,
                   verbose, **kw)


def Stokes2D0(nx=None, ny=None, return_solver=False, verbose=False, **kw):
    """scripts/previous_damp/Stokes2D0.jl:72-173 (2D viscous, damped scheme; NX, NY default 511)."""
    return _script("2d_v_damp", nx or _env("NX", 511), ny or _env("NY", 511), None, return_solver, verbose, **kw)


def Stokes2D_ve0(nx=None, ny=None, return_solver=False, verbose=False, **kw):
    """scripts/previous_damp/Stokes2D_ve0.jl:82-204 (2D Maxwell VE, damped scheme, 5 steps)."""
    return _script("2d_ve_damp", nx or _env("NX", 511), ny or _env("NY", 511), None, return_solver, verbose, **kw)


def Stokes3D0(nx=None, ny=None, nz=None, return_solver=False, verbose=False, **kw):
    """scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl:96-248 on one rank (3D viscous,
    damped scheme; NX, NY, NZ default 63)."""
    return _script("3d_v_damp", nx or _env("NX", 63), ny or _env("NY", 63), nz or _env("NZ", 63), return_solver,
                   verbose, **kw)


# Effective memory traffic per PT iteration, in bytes, by the reference's own
# convention (A_eff; Stokes3D_ve_perf.jl:229, Stokes2D_ve_perf.jl:173).
def a_eff_bytes(variant, nx, ny, nz=1, itemsize=8):
    return output.A_EFF_ARRAYS[variant] * nx * ny * (nz if variant.startswith("3d") else 1) * itemsize
