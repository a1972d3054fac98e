"""Solver: one PT Stokes problem on the GPU, driven through the C ABI.

The methods carry the reference's kernel-role names (compute_P!, compute_τ!,
compute_dV!, compute_V!, compute_Pt_τ!, compute_Res!, assign_τ!, bc_*!) and act on the
fields the context owns on the device. Fields cross to and from the host as Float64
column-major numpy arrays with the reference's own extents.
"""
import ctypes
import math

import numpy as np

from . import _abi
from ._abi import FIELD_ID, PtsCheck, PtsDesc, PtsSolveInfo, check

PI = math.pi

# Physics and numerics of each script (the constants at the top of Stokes2D_()/Stokes3D_()).
VARIANT_DEFAULTS = {
    # scripts/Stokes2D.jl:74-84
    "2d_v": dict(nt=1, iter_max=1e5, nout=500, eps=1e-8, CFL=0.9 / math.sqrt(2), Re=5 * PI, r=1.0),
    # scripts/Stokes2D_ve.jl:89-103
    "2d_ve": dict(nt=5, iter_max=2e5, nout=200, eps=1e-8, CFL=0.8 / math.sqrt(2), Re=5 * PI, r=1.0),
    # scripts/Stokes2D_ve_perf.jl:82-97
    "2d_ve_perf": dict(nt=1, iter_max=100, nout=2000, eps=1e-8, CFL=0.8 / math.sqrt(2), Re=5 * PI, r=1.0),
    # scripts/stokes_3D/Stokes3D_ve_multixpu.jl:120-134
    "3d_ve": dict(nt=5, iter_max=2e5, nout=200, eps=1e-8, CFL=0.8 / math.sqrt(3), Re=6 * PI, r=1.0),
    # scripts/stokes_3D/Stokes3D_ve_perf.jl:118-132
    "3d_ve_perf": dict(nt=1, iter_max=200, nout=2000, eps=1e-8, CFL=0.8 / math.sqrt(3), Re=6 * PI, r=1.0),
    # 3D viscous (no script): the 3D numerics, one "time step"
    "3d_v": dict(nt=1, iter_max=2e5, nout=200, eps=1e-8, CFL=0.8 / math.sqrt(3), Re=6 * PI, r=1.0),
    # scripts/previous_damp/Stokes2D0.jl:76-86 (damped scheme; r, Re, CFL unused)
    "2d_v_damp": dict(nt=1, iter_max=1e5, nout=500, eps=1e-8, CFL=0.0, Re=0.0, r=0.0, Vdmp=4.0, beta_n=2.0,
                      Vsc=1.0, Ptsc=3.0),
    # scripts/previous_damp/Stokes2D_ve0.jl:91-99
    "2d_ve_damp": dict(nt=5, iter_max=2e5, nout=200, eps=1e-8, CFL=0.0, Re=0.0, r=0.0, Vdmp=4.0, beta_n=2.0,
                       Vsc=1.0, Ptsc=3.0),
    # scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl:102-109 (one solve)
    "3d_v_damp": dict(nt=1, iter_max=6e4, nout=500, eps=1e-8, CFL=0.0, Re=0.0, r=0.0, Vdmp=4.0, beta_n=3.0,
                      Vsc=1.0, Ptsc=5.0),
}
DAMPING = ("Vdmp", "beta_n", "Vsc", "Ptsc")


def linrange(a, b, n):
    """Values of Julia's ``LinRange(a, b, n)``: (1-t)*a + t*b, t = (i-1)/(n-1)."""
    d = n - 1
    return np.array([(1 - (j / d)) * a + (j / d) * b if d > 0 else a for j in range(n)])


class Solver:
    """A PT Stokes context (``pts_ctx``) with its device fields.

    ``variant`` is one of ``2d_v, 2d_ve, 2d_ve_perf, 3d_ve, 3d_ve_perf, 3d_v, 2d_v_damp,
    2d_ve_damp, 3d_v_damp``.
    Keyword arguments override the script defaults (``VARIANT_DEFAULTS``) and the
    physics (``lx, ly, lz, G, xi, mus0``: ``dt = mus0/(G*xi)`` as in the scripts).
    """

    def __init__(self, variant, nx, ny, nz=None, precision="fp64", lib=None, **kw):
        self.lib = lib or _abi.load()
        self.variant = variant
        self.ndim = 3 if variant.startswith("3d") else 2
        p = dict(lx=10.0, ly=10.0, lz=10.0, xi=1.0, mus0=1.0, G=1.0, max_l=0.0, mixed_inner=0, single_pass=0,
                 adjoint=0, stencil=0, stencil_tile=0, stencil_kz=0, stencil_vtile=0, mixed_sweep=0)
        p.update(VARIANT_DEFAULTS[variant])
        p.update(kw)
        self.p = p
        self.nx, self.ny, self.nz = nx, ny, (nz if self.ndim == 3 else 1)
        self.dt = p["mus0"] / (p["G"] * p["xi"])
        d = PtsDesc()
        d.variant = _abi.VARIANTS[variant]
        d.precision = _abi.PRECISIONS[precision]
        d.nx, d.ny, d.nz = nx, ny, (nz if self.ndim == 3 else 1)
        d.nout = int(p["nout"])
        d.lx, d.ly, d.lz = p["lx"], p["ly"], p["lz"]
        d.G, d.dt = p["G"], self.dt
        d.r, d.Re, d.CFL = p["r"], p["Re"], p["CFL"]
        d.max_l, d.eps, d.iter_max = p["max_l"], p["eps"], float(p["iter_max"])
        d.mixed_inner = int(p["mixed_inner"])
        d.single_pass = int(p["single_pass"])
        d.adjoint = int(p["adjoint"])
        d.stencil = int(p["stencil"])
        d.stencil_tile = int(p["stencil_tile"])
        d.stencil_kz = int(p["stencil_kz"])
        d.stencil_vtile = int(p["stencil_vtile"])
        d.mixed_sweep = int(p["mixed_sweep"])
        self.desc = d
        ctx = ctypes.c_void_p()
        check(self.lib, None, self.lib.pts_create(ctypes.byref(d), ctypes.byref(ctx)))
        self.ctx = ctx
        if variant.endswith("_damp"):
            self.set_damping(*(p[k] for k in DAMPING))
        self.dx = p["lx"] / nx
        self.dy = p["ly"] / ny
        self.dz = p["lz"] / nz if self.ndim == 3 else 1.0

    # ---------------------------------------------------------------- lifetime
    def close(self):
        if getattr(self, "ctx", None):
            self.lib.pts_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, rc):
        return check(self.lib, self.ctx, rc)

    # ---------------------------------------------------------------- fields
    def shape(self, name):
        s = (ctypes.c_int64 * 3)()
        self._ck(self.lib.pts_field_shape(self.ctx, FIELD_ID[name], s))
        return tuple(s[: self.ndim])

    def get(self, name):
        shp = self.shape(name)
        out = np.empty(shp, dtype=np.float64, order="F")
        self._ck(self.lib.pts_get_field(self.ctx, FIELD_ID[name], out.ctypes.data, out.size))
        return out

    def set(self, name, a):
        a = np.asfortranarray(a, dtype=np.float64)
        if a.shape != self.shape(name):
            raise ValueError(f"{name}: expected shape {self.shape(name)}, got {a.shape}")
        self._ck(self.lib.pts_set_field(self.ctx, FIELD_ID[name], a.ctypes.data, a.size))

    def set_device(self, name, ptr, n):
        self._ck(self.lib.pts_set_field_device(self.ctx, FIELD_ID[name], ptr, n))

    def get_device(self, name, ptr, n):
        self._ck(self.lib.pts_get_field_device(self.ctx, FIELD_ID[name], ptr, n))

    # ---------------------------------------------------------------- set-up
    def init_inclusion(self, mus0=1.0, musi=1e-3, radius2=1.0, ebg=1.0):
        self._ck(self.lib.pts_init_inclusion(self.ctx, mus0, musi, radius2, ebg))

    def init_inclusions(self, rows, mus0=1.0, ebg=1.0):
        """create_inclusions! (Stokes2D_param.jl:83-99) on the device for a list of inclusions:
        ``rows`` is (count, 5) [x, y, z, r2, mus], centres relative to the domain centre
        (``ptstokes.adjoint.inclusion_array``); the first inclusion a cell centre is inside
        gives its viscosity, else mus0. Velocities get the pure-shear ICs, the rest zero."""
        rows = np.asarray(rows, dtype=np.float64).reshape(-1, 5)
        arr = (_abi.PtsInclusion * max(len(rows), 1))()
        for q, (x, y, z, r2, mu) in enumerate(rows):
            arr[q] = _abi.PtsInclusion(x, y, z, r2, mu)
        self._ck(self.lib.pts_init_inclusions(self.ctx, arr, len(rows), mus0, ebg))

    def smooth(self, nsweeps=10, fact=1.0):
        self._ck(self.lib.pts_smooth(self.ctx, nsweeps, fact))

    def compute_maxloc(self):
        self._ck(self.lib.pts_compute_maxloc(self.ctx))

    def compute_iter_params(self):
        self._ck(self.lib.pts_compute_iter_params(self.ctx))

    def set_damping(self, Vdmp=4.0, beta_n=None, Vsc=1.0, Ptsc=None):
        """Numerics of the damped scheme (Stokes2D_ve0.jl:95-98, Stokes3D0_multixpu.jl:105-108);
        before compute_iter_params. β_n and Ptsc default to the script's (2, 3 in 2D; 3, 5 in 3D)."""
        if beta_n is None:
            beta_n = 3.0 if self.ndim == 3 else 2.0
        if Ptsc is None:
            Ptsc = 5.0 if self.ndim == 3 else 3.0
        self._ck(self.lib.pts_set_damping(self.ctx, Vdmp, beta_n, Vsc, Ptsc))
        self.p.update(Vdmp=Vdmp, beta_n=beta_n, Vsc=Vsc, Ptsc=Ptsc)

    def setup_inclusion(self, musi=1e-3, radius2=1.0, ebg=1.0, nsmooth=10):
        """The scripts' set-up: ICs, 10x smooth!, maxloc + bc, iteration parameters."""
        self.init_inclusion(self.p["mus0"], musi, radius2, ebg)
        self.smooth(nsmooth, 1.0)
        self.compute_maxloc()
        self.compute_iter_params()
        return self

    # ---------------------------------------------------------------- roles
    def assign_tau(self):
        self._ck(self.lib.pts_assign_tau(self.ctx))

    def compute_P(self):
        self._ck(self.lib.pts_compute_P(self.ctx))

    def compute_tau(self):
        self._ck(self.lib.pts_compute_tau(self.ctx))

    def compute_dV(self):
        self._ck(self.lib.pts_compute_dV(self.ctx))

    def compute_V(self):
        self._ck(self.lib.pts_compute_V(self.ctx))

    def apply_bc(self):
        self._ck(self.lib.pts_apply_bc(self.ctx))

    def compute_Pt_tau(self):
        self._ck(self.lib.pts_compute_Pt_tau(self.ctx))

    def compute_V_bc(self):
        self._ck(self.lib.pts_compute_V_bc(self.ctx))

    def set_kernel_timing(self, on=True):
        """A CUDA event after each kernel of every block of PT iterations (graph blocks too)."""
        self._ck(self.lib.pts_set_kernel_timing(self.ctx, 1 if on else 0))

    def kernel_times(self, cap=1 << 16):
        """Elapsed ms between the events of the last block, in launch order (synchronous)."""
        buf = (ctypes.c_float * cap)()
        cnt = ctypes.c_int64()
        self._ck(self.lib.pts_kernel_times(self.ctx, buf, cap, ctypes.byref(cnt)))
        return list(buf[: min(cnt.value, cap)])

    def compute_res(self):
        c = PtsCheck()
        self._ck(self.lib.pts_compute_res(self.ctx, ctypes.byref(c)))
        return c.as_dict()

    # ---------------------------------------------------------------- adjoint (3d_v)
    def apply_operator(self):
        """τ = 2·Mus·ε̇(V), then Rx, Ry, Rz and ∇V of the current fields: one application of the
        forward operator, or of its transpose for a context created with adjoint=1."""
        c = PtsCheck()
        self._ck(self.lib.pts_apply_operator(self.ctx, ctypes.byref(c)))
        return c.as_dict()

    def gradient_logmu(self, adj, add=False):
        """∂J/∂log μ into this (forward) context's "grad" field from the adjoint context adj
        (add=True adds one visco-elastic step's term)."""
        fn = self.lib.pts_gradient_logmu_add if add else self.lib.pts_gradient_logmu
        self._ck(fn(self.ctx, adj.ctx))

    # ---------------------------------------------------------------- kernel form
    def set_stencil(self, stencil=0, tile=0, kz=0, vtile=0):
        """Kernel form of compute_Pt_τ! and compute_V! + bc (pts_set_stencil): 0 = z-marching
        with TMA-staged planes (tile configurations `tile` and `vtile`, `kz` planes per block),
        1 = one thread per cell or face."""
        self._ck(self.lib.pts_set_stencil(self.ctx, int(stencil), int(tile), int(kz), int(vtile)))
        d = self.desc
        d.stencil, d.stencil_tile, d.stencil_kz, d.stencil_vtile = int(stencil), int(tile), int(kz), int(vtile)

    def tune_stencil(self, iters=20, kzs=(16, 32, 64), use_cache=True):
        """Time every z-marching (2D: y-marching) tile configuration x planes-per-block (2D: rows
        per block) in `kzs` on this problem
        (`iters` PT iterations each, CUDA events on the context's stream), keep the fastest,
        and cache the choice per (variant, precision, grid) in ~/.cache/ptstokes/stencil.json.
        The iterations advance the fields; results do not depend on the configuration."""
        import json
        import os
        import time

        import torch

        key = f"{self.variant}/{self.desc.precision}/{self.nx}x{self.ny}x{self.nz}"
        path = os.path.join(os.path.expanduser("~"), ".cache", "ptstokes", "stencil.json")
        cache = {}
        if use_cache and os.path.exists(path):
            try:
                cache = json.load(open(path))
            except Exception:
                cache = {}
        if use_cache and key in cache:
            e = cache[key]
            self.set_stencil(0, e["tile"], e["kz"], e.get("vtile", 0))
            return e
        stream = torch.cuda.ExternalStream(self.stream_handle())

        def timed(tile, kz, vtile):
            self.set_stencil(0, tile, kz, vtile)
            self.iterate(2)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            self.iterate(iters)
            b.record(stream)
            b.synchronize()
            return a.elapsed_time(b) / iters

        # compute_Pt_τ! tiles x z-chunks (2D: rows per block) with the default compute_V! tile,
        # then the V tiles (3D only: 2D compute_V! has one form)
        ntiles = (self.lib.pts_stencil_tiles(self.desc.precision) if self.ndim == 3
                  else self.lib.pts_stencil_tiles_2d())
        ms = {f"{t}:{kz}:0": timed(t, kz, 0) for t in range(ntiles) for kz in kzs}
        tile, kz, _ = map(int, min(ms, key=ms.get).split(":"))
        nv = self.lib.pts_stencil_vtiles(self.desc.precision) if self.ndim == 3 else 1
        for v in range(1, nv):
            ms[f"{tile}:{kz}:{v}"] = timed(tile, kz, v)
        tile, kz, vtile = map(int, min(ms, key=ms.get).split(":"))
        self.set_stencil(0, tile, kz, vtile)
        entry = {"tile": tile, "kz": kz, "vtile": vtile, "ms_per_iteration": ms, "when": time.time()}
        if use_cache:
            try:
                os.makedirs(os.path.dirname(path), exist_ok=True)
                cache[key] = entry
                json.dump(cache, open(path, "w"), indent=1)
            except OSError:
                pass
        return entry

    # ---------------------------------------------------------------- drivers
    def iterate(self, n):
        self._ck(self.lib.pts_iterate(self.ctx, int(n)))

    def stream_handle(self):
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        h = ctypes.c_void_p()
        self._ck(self.lib.pts_stream(self.ctx, ctypes.byref(h)))
        return h.value or 0

    def sync(self):
        self._ck(self.lib.pts_sync(self.ctx))

    def solve(self):
        info = PtsSolveInfo()
        self._ck(self.lib.pts_solve(self.ctx, ctypes.byref(info)))
        return dict(iters=info.iters, converged=bool(info.converged), nchecks=info.nchecks, last=info.last.as_dict())

    def run(self, nt=None):
        nt = self.p["nt"] if nt is None else nt
        per = (ctypes.c_int64 * max(nt, 1))()
        info = PtsSolveInfo()
        self._ck(self.lib.pts_run(self.ctx, nt, per, ctypes.byref(info)))
        return dict(ittot=info.iters, iters=list(per[:nt]), converged=bool(info.converged), last=info.last.as_dict())

    # ---------------------------------------------------------------- grid
    def centres(self):
        """xc, yc[, zc] = LinRange(dx/2, lx-dx/2, nx), ... (Stokes3D_ve_perf.jl:139)."""
        p = self.p
        out = [linrange(self.dx / 2, p["lx"] - self.dx / 2, self.nx), linrange(self.dy / 2, p["ly"] - self.dy / 2, self.ny)]
        if self.ndim == 3:
            out.append(linrange(self.dz / 2, p["lz"] - self.dz / 2, self.nz))
        return out
