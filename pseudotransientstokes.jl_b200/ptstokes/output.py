"""The reference scripts' output files, written from a solved context.

Each script appends one whitespace-separated line per run to ``output/out_<script>.txt``
(the columns its Matlab readers parse with ``fscanf``, e.g. visu/viz_perf_stokes.m:4-11)
and, with DO_SAVE_VIZ, dumps a few fields to ``out_visu/<name>.mat``:

    script                     line (source)                                        MAT fields
    Stokes2D.jl                nx ny iter (:164-165)                                --
    Stokes2D_ve.jl             nx ny ittot nt (:197-198)                            Pt_2D Mus_2D Txy_2D Vy_2D dx_2D dy_2D (:203)
    Stokes2D_ve_perf.jl        nx ny ittot t_toc A_eff t_it T_eff (:189-190)        same as Stokes2D_ve.jl (:195)
    Stokes3D_ve_multixpu.jl    nx ny nz ittot nt (:285-286)                         Pt_3D Mus_3D Txz_3D Vz_3D dx_3D dy_3D dz_3D (:291)
    Stokes3D_ve_perf.jl        1 nx ny nz ittot wtime A_eff wtime_it T_eff (:244-247) same as the multi-XPU script (:250)
    previous_damp/Stokes2D0.jl     nx ny iter (:168-169)                            --
    previous_damp/Stokes2D_ve0.jl  nx ny ittot nt (:195-196)                        same as Stokes2D_ve.jl (:199-200)
    stokes_3D/previous_damp/Stokes3D0_multixpu.jl  nx ny nz iter (:241-243)         --

Numbers are printed as Julia prints them (``println`` of an Int or a Float64: shortest
round-trip digits, scientific below 1e-4 and from 1e6 upward), so the lines read like the
reference's own. The MAT files are MATLAB v5 (scipy), which MATLAB's ``load`` reads like
the v7.3 files MAT.jl writes. Timings: ``t_it = wtime/(ittot - 10)`` as in the scripts, with
wtime the run's whole wall time (the scripts start their clock at iteration 11).
"""
import os
from decimal import Decimal

import numpy as np

# A_eff arrays per PT iteration of each script (the scripts' own conventions)
A_EFF_ARRAYS = {"2d_v": 6, "2d_ve": 13, "2d_ve_perf": 18, "3d_ve": 21, "3d_ve_perf": 29, "3d_v": 23,
                "2d_v_damp": 6, "2d_ve_damp": 13, "3d_v_damp": 8}


def jl(x):
    """`string(x)` of Julia for an Int or a Float64."""
    if isinstance(x, (int, np.integer)):
        return str(int(x))
    x = float(x)
    if x == 0.0:
        return "-0.0" if np.signbit(x) else "0.0"
    if not np.isfinite(x):
        return "NaN" if np.isnan(x) else ("Inf" if x > 0 else "-Inf")
    sign, digits, exp = Decimal(repr(x)).as_tuple()
    digits = list(digits)
    while len(digits) > 1 and digits[-1] == 0:
        digits.pop()
        exp += 1
    s = "-" if sign else ""
    e10 = len(digits) - 1 + exp  # scientific exponent
    ds = "".join(map(str, digits))
    if e10 < -4 or e10 > 5:
        return f"{s}{ds[0]}.{ds[1:] or '0'}e{e10}"
    if exp >= 0:
        return f"{s}{ds}{'0' * exp}.0"
    point = len(ds) + exp
    if point > 0:
        return f"{s}{ds[:point]}.{ds[point:]}"
    return f"{s}0.{'0' * (-point)}{ds}"


def _append(path, values):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "a") as fh:
        fh.write(" ".join(jl(v) for v in values) + "\n")


LINE_FILES = {"2d_v": "out_Stokes2D.txt", "2d_ve": "out_Stokes2D_ve.txt", "2d_ve_perf": "out_Stokes2D_ve_perf.txt",
              "3d_ve": "out_Stokes3D_ve.txt", "3d_ve_perf": "out_Stokes3D_ve_perf.txt", "3d_v": "out_Stokes3D_v.txt",
              "2d_v_damp": "out_Stokes2D0.txt", "2d_ve_damp": "out_Stokes2D_ve0.txt", "3d_v_damp": "out_Stokes3D0.txt"}
MAT_FILES = {"2d_ve": "Stokes_2D_ve.mat", "2d_ve_perf": "Stokes_2D_ve_perf.mat", "3d_ve": "Stokes_3D_ve.mat",
             "3d_ve_perf": "Stokes_3D_ve_perf.mat", "3d_v": "Stokes_3D_v.mat", "2d_ve_damp": "Stokes_2D_ve0.mat"}


def result_line(variant, nx, ny, nz, ittot, nt, wtime):
    """The values of the script's output line (see the table above)."""
    n = nx * ny * (nz or 1)
    a_eff = A_EFF_ARRAYS[variant] * n * 8 / 1e9
    t_it = wtime / max(ittot - 10, 1)
    t_eff = a_eff / t_it
    if variant in ("2d_v", "2d_v_damp"):
        return [nx, ny, ittot]
    if variant in ("2d_ve", "2d_ve_damp"):
        return [nx, ny, ittot, nt]
    if variant == "2d_ve_perf":
        return [nx, ny, ittot, wtime, a_eff, t_it, t_eff]
    if variant == "3d_ve":
        return [nx, ny, nz, ittot, nt]
    if variant == "3d_v_damp":
        return [nx, ny, nz, ittot]
    return [1, nx, ny, nz, ittot, wtime, a_eff, t_it, t_eff]


def save_line(solver, res, wtime, outdir="output"):
    """Append the script's line for a finished run (`res` from Solver.run())."""
    values = result_line(solver.variant, solver.nx, solver.ny, solver.nz if solver.ndim == 3 else None,
                         res["ittot"], len(res["iters"]), wtime)
    path = os.path.join(outdir, LINE_FILES[solver.variant])
    _append(path, values)
    return path


def save_visu(solver, outdir="out_visu"):
    """The script's MAT dump: Pt, Mus, τxy/Vy (2D) or τxz/Vz (3D) and the grid spacings."""
    from scipy.io import savemat

    if solver.variant not in MAT_FILES:
        raise ValueError(f"{solver.variant}: the reference script writes no MAT file")
    if solver.ndim == 2:
        d = {"Pt_2D": solver.get("Pt"), "Mus_2D": solver.get("Mus"), "Txy_2D": solver.get("txy"),
             "Vy_2D": solver.get("Vy"), "dx_2D": solver.dx, "dy_2D": solver.dy}
    else:
        d = {"Pt_3D": solver.get("Pt"), "Mus_3D": solver.get("Mus"), "Txz_3D": solver.get("txz"),
             "Vz_3D": solver.get("Vz"), "dx_3D": solver.dx, "dy_3D": solver.dy, "dz_3D": solver.dz}
    os.makedirs(outdir, exist_ok=True)
    path = os.path.join(outdir, MAT_FILES[solver.variant])
    savemat(path, d, do_compression=True)
    return path
