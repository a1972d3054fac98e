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
    Stokes2D_ve_param   scripts/Stokes2D_ve_param.jl (aspect-ratio study); aspect_ratio_sweep is
                        scripts/runme_Stokes2D_aspect_ratio.jl's loop over its parameters
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


def length_error(s, chk):
    """The error measure the 2D scripts keep commented out beside their check
    (Stokes2D_ve0.jl:166, Stokes2D0.jl:145, Stokes2D.jl:142): max of ||Rx||/length(Rx),
    ||Ry||/length(Ry), ||∇V||/length(∇V). It is recovered from a check `chk` of context `s`
    (pts_compute_res: norm_R = ||R|| / (Pmax-Pmin) * lx / sqrt(length(R)), norm_∇V likewise
    with Vmax-Vmin and the context's default norm scale lx)."""
    import math

    if s.ndim != 2:
        raise ValueError("length_error restates the 2D scripts' measure")
    nx, ny, lx = s.nx, s.ny, s.p["lx"]
    lens = ((nx - 1) * (ny - 2), (nx - 2) * (ny - 1), nx * ny)
    dP, dV = chk["Pmax"] - chk["Pmin"], chk["Vmax"] - chk["Vmin"]
    norms = [chk["norm_Rx"] * dP * math.sqrt(lens[0]) / lx / lens[0],
             chk["norm_Ry"] * dP * math.sqrt(lens[1]) / lx / lens[1],
             chk["norm_divV"] * dV * math.sqrt(lens[2]) / lx / lens[2]]
    if any(math.isnan(v) for v in norms):
        return float("nan"), norms
    return max(norms), norms


def run_length_error(s, nt=None):
    """The scripts' time loop with the check's commented-out error measure (`length_error`),
    driven from the host through the context's own calls: per physical step `assign_τ!`,
    then `while err > ε && iter <= iterMax` in blocks of PT iterations that end on the
    multiples of nout, where the check runs (Stokes2D_ve0.jl:147-175). The damped rates
    carry over between steps, as in the script. With it, `Stokes2D_ve0` takes the
    iteration totals of the reference's output/out_Stokes2D_ve0.txt."""
    import math

    p = s.p
    nt = p["nt"] if nt is None else nt
    eps, nout, iter_max = p["eps"], int(p["nout"]), math.floor(float(p["iter_max"]))
    if nout < 1:
        raise ValueError("nout must be >= 1: the check runs every nout PT iterations")
    iters, err = [], 2 * eps
    for _ in range(nt):
        err, it = 2 * eps, 0
        if s.variant != "2d_v_damp":
            s.assign_tau()
        while err > eps and it <= iter_max:
            k = min(nout - it % nout, iter_max - it + 1)  # up to the next check or past iterMax
            s.iterate(k)
            it += k
            if it % nout == 0:
                err, _ = length_error(s, s.compute_res())
                if math.isnan(err):
                    raise FloatingPointError("NaN")
        iters.append(it)
    return dict(ittot=sum(iters), iters=iters, converged=not (err > eps), err=err)


def _script(variant, nx, ny, nz, return_solver, verbose, do_save=None, do_save_viz=None, err_form="scaled",
            **kw):
    if err_form not in ("scaled", "length"):
        raise ValueError(f"err_form must be 'scaled' or 'length', not {err_form!r}")
    if err_form == "length" and variant not in ("2d_ve_damp", "2d_v_damp"):
        raise ValueError("err_form='length' is the damped 2D scripts' alternative check")
    s = Solver(variant, nx, ny, nz, **kw)
    s.setup_inclusion(musi=kw.get("musi", 1e-3))
    t0 = time.perf_counter()
    res = s.run() if err_form == "scaled" else run_length_error(s)
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
    """scripts/previous_damp/Stokes2D_ve0.jl:82-204 (2D Maxwell VE, damped scheme, 5 steps).
    err_form="length" checks with the script's commented-out measure (:166), the one its
    published totals (output/out_Stokes2D_ve0.txt) were taken with."""
    return _script("2d_ve_damp", nx or _env("NX", 511), ny or _env("NY", 511), None, return_solver, verbose, **kw)


def Stokes3D0(nx=None, ny=None, nz=None, return_solver=False, verbose=False, **kw):
    """scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl:96-248 on one rank (3D viscous,
    damped scheme; NX, NY, NZ default 63)."""
    return _script("3d_v_damp", nx or _env("NX", 63), ny or _env("NY", 63), nz or _env("NZ", 63), return_solver,
                   verbose, **kw)


def ve_param_solver(ny, nsub=1, fact=1.0, ly=10.0, lib=None, **kw):
    """The context of scripts/Stokes2D_ve_param.jl: ly = 10, lx = nsub*ly, nx = nsub*(ny+1)-1
    (:99-107); CFL 0.87/sqrt(2), eps = 1e-6, iterMax = 100nx, nout = nx (:103-109);
    min_lxy = fact*min(lx,ly) as the length of the iteration parameters (:110, :150); norm_Rx
    scaled by lx, norm_Ry and norm_∇V by ly (:175-177). Set up as the script does: pure-shear
    velocities, nsub inclusions of radius 1 centred at (isub-1)*ly + ly/2 along x (built on the
    host as the script builds it, :138-141), 10 smooth! sweeps, maxloc, iteration parameters."""
    import math

    import numpy as np

    lx = nsub * ly
    nx = nsub * (ny + 1) - 1
    p = dict(lx=lx, ly=ly, CFL=0.87 / math.sqrt(2), eps=1e-6, iter_max=100 * nx, nout=nx, nt=5,
             max_l=fact * min(lx, ly))
    p.update(kw)
    s = Solver("2d_ve", nx, ny, lib=lib, **p)
    s._ck(s.lib.pts_set_norm_scales(s.ctx, lx, ly, 1.0, ly))
    dx, dy = lx / nx, ly / ny
    ix = np.arange(1, nx + 1, dtype=np.float64)
    iy = np.arange(1, ny + 1, dtype=np.float64)
    mus = np.ones((nx, ny), order="F")
    for isub in range(1, nsub + 1):
        X = (ix - 1) * dx + 0.5 * dx - 0.5 * ly - (isub - 1) * ly
        Y = (iy - 1) * dy + 0.5 * dy - 0.5 * ly
        mus[(X[:, None] ** 2 + Y[None, :] ** 2) < 1.0] = 1e-3
    s.init_inclusion(1.0, 1.0, 0.0, 1.0)  # pure shear, every other field zero
    s.set("Mus", mus)
    s.smooth(10, 1.0)
    s.compute_maxloc()
    s.compute_iter_params()
    s.nsub, s.fact = nsub, fact
    return s


def Stokes2D_ve_param(ny=None, nsub=None, fact=None, return_solver=False, verbose=False, **kw):
    """scripts/Stokes2D_ve_param.jl:87-212: 5 Maxwell steps of the aspect-ratio problem (RESOL,
    NSUB, FACT from the environment as the script reads them). Returns (xc, yc, Pt) and, with
    return_solver, the solver and its outcome, including the script's output line
    ``nx ny nsub fact ittot nt err``."""
    ny = ny or _env("RESOL", 255)
    nsub = nsub or _env("NSUB", 1)
    fact = fact if fact is not None else float(os.environ.get("FACT", "1.0"))
    s = ve_param_solver(ny, nsub, fact, **kw)
    t0 = time.perf_counter()
    res = s.run()
    res["wall_s"] = time.perf_counter() - t0
    res["line"] = f"{s.nx} {s.ny} {nsub} {fact} {res['ittot']} {len(res['iters'])} {res['last']['err']}"
    if verbose:
        print(res["line"])
    out = (*s.centres(), s.get("Pt"))
    if return_solver:
        return out, s, res
    s.close()
    return out


def aspect_ratio_sweep(facts=(1.0, 0.9, 0.8, 0.7, 0.6, 0.5, 0.4, 0.3, 0.2, 0.1), nsubs=(1, 2, 4, 8),
                       resols=(127, 255, 511, 1023, 2047), in_flight=4, lib=None):
    """scripts/runme_Stokes2D_aspect_ratio.jl: Stokes2D_ve_param for the Cartesian product of
    FACT x NSUB x RESOL (the reference starts one Julia process per instance). Here up to
    `in_flight` contexts iterate at once, one host thread each (the C calls release the GIL),
    on their own streams. Returns one result per instance, in the reference's loop order, with
    the script's output line."""
    import itertools
    import threading

    jobs = list(itertools.product(facts, nsubs, resols))
    out = [None] * len(jobs)
    nxt = [0]
    lock = threading.Lock()
    errors = []

    def worker():
        while True:
            with lock:
                q = nxt[0]
                nxt[0] += 1
            if q >= len(jobs) or errors:
                return
            fact, nsub, ny = jobs[q]
            try:
                s = ve_param_solver(ny, nsub, fact, lib=lib)
                res = s.run()
                res["line"] = f"{s.nx} {s.ny} {nsub} {fact} {res['ittot']} {len(res['iters'])} {res['last']['err']}"
                res.update(fact=fact, nsub=nsub, ny=ny, nx=s.nx)
                s.close()
                out[q] = res
            except Exception as e:  # re-raised below
                errors.append(e)

    threads = [threading.Thread(target=worker) for _ in range(max(1, in_flight))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return out


# Effective memory traffic per PT iteration, in bytes, by the reference's own
# convention (A_eff; Stokes3D_ve_perf.jl:229, Stokes2D_ve_perf.jl:173).
def a_eff_bytes(variant, nx, ny, nz=1, itemsize=8):
    return output.A_EFF_ARRAYS[variant] * nx * ny * (nz if variant.startswith("3d") else 1) * itemsize
