"""Batched 2D viscous sweeps: many uneven instances in one persistent GPU launch.

The reference runs its parameter sweeps as one Julia process per instance
(scripts/runme_Stokes2D_shear_weak.jl:1-26, runme_Stokes2D_gravity_weak.jl:1-26,
runme_Stokes2D_aspect_ratio.jl:1-24). ``Batch`` runs a whole sweep in one cooperative
launch with per-instance convergence (``pts_batch_*`` in include/ptstokes.h);
``sweep_instances`` draws the seeded sweep of 256 instances; ``autotune`` picks the tile
shape by timing the candidates on the batch itself and caches the choice.
"""
import ctypes
import json
import math
import os
import time

import numpy as np

from . import _abi
from ._abi import FIELD_ID, PtsBatchDesc, PtsBatchInstance, PtsBatchVEInstance

TILE_SHAPES = [(32, 4), (32, 8), (64, 4), (32, 16)]


def sweep_instances(n=256, seed=1855, sizes=(63, 127, 255, 511), ly=10.0):
    """The seeded sweep: nx in `sizes`, lx/ly ~ U[1,4] (ly = 10, ny so that dy ~ dx), one
    centred inclusion of radius 1 with log10 viscosity contrast ~ U[-6,-1], and either
    buoyancy-driven (inclusion Δρg = 1, no background flow) or pure shear (εbg = 1), 50/50."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(rng.choice(sizes))
        aspect = float(rng.uniform(1.0, 4.0))
        lx = aspect * ly
        ny = max(15, int(round((nx + 1) / aspect)) - 1)
        musi = float(10.0 ** rng.uniform(-6.0, -1.0))
        gravity = bool(rng.random() < 0.5)
        out.append(dict(nx=nx, ny=ny, lx=lx, ly=ly, musi=musi, radius2=1.0,
                        rhogi=1.0 if gravity else 0.0, ebg=0.0 if gravity else 1.0))
    return out


class Batch:
    def __init__(self, instances, nout=200, eps=1e-8, iter_max=0, tile=1, r=1.0, Re=5 * math.pi,
                 CFL=0.9 / math.sqrt(2), lib=None):
        """`iter_max` <= 0 gives each instance the sweep script's iterMax = 100max(nx,ny)
        (scripts/Stokes2D_param.jl:146); a positive value is a common iterMax."""
        self.lib = lib or _abi.load()
        self.instances = [dict(d) for d in instances]
        n = len(self.instances)
        arr = (PtsBatchInstance * n)()
        for q, d in enumerate(self.instances):
            arr[q] = PtsBatchInstance(d["nx"], d["ny"], d["lx"], d["ly"], d["musi"], d.get("radius2", 1.0),
                                      d.get("rhogi", 0.0), d.get("ebg", 1.0))
        desc = PtsBatchDesc()
        desc.nout, desc.tile, desc.eps, desc.iter_max = nout, tile, eps, float(iter_max)
        desc.r, desc.Re, desc.CFL = r, Re, CFL
        self.desc = desc
        h = ctypes.c_void_p()
        rc = self.lib.pts_batch_create(ctypes.byref(desc), arr, n, ctypes.byref(h))
        if rc != 0:
            raise _abi.PtsError(rc, (self.lib.pts_last_error(None) or b"").decode())
        self.h = h
        self.n = n
        self.tile = tile

    def _ck(self, rc):
        if rc != 0:
            raise _abi.PtsError(rc, (self.lib.pts_batch_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.pts_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup(self):
        self._ck(self.lib.pts_batch_setup(self.h))
        return self

    def set_tile(self, tile):
        self._ck(self.lib.pts_batch_set_tile(self.h, int(tile)))
        self.tile = int(tile)

    def stream_handle(self):
        s = ctypes.c_void_p()
        self._ck(self.lib.pts_batch_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def solve(self, iter_limit=-1, raise_on_nan=True):
        """Run the sweep. An instance whose check gives NaN is frozen there (converged False);
        with raise_on_nan the call then raises PtsError(PTS_E_NAN), else the result has
        nan=True and the other instances' outcomes stand."""
        n = self.n
        iters = (ctypes.c_int64 * n)()
        err = (ctypes.c_double * n)()
        conv = (ctypes.c_int32 * n)()
        graph = ctypes.c_int32()
        rc = self.lib.pts_batch_solve(self.h, int(iter_limit), iters, err, conv, ctypes.byref(graph))
        if rc != 0 and (raise_on_nan or rc != _abi.PTS_E_NAN):
            self._ck(rc)
        return dict(iters=list(iters), err=list(err), converged=[bool(c) for c in conv], used_graph=bool(graph.value),
                    nan=rc == _abi.PTS_E_NAN)

    def shape(self, q, name):
        nx, ny = self.instances[q]["nx"], self.instances[q]["ny"]
        return {"Vx": (nx + 1, ny), "Vy": (nx, ny + 1), "txy": (nx - 1, ny - 1), "Rx": (nx - 1, ny - 2),
                "Ry": (nx - 2, ny - 1)}.get(name, (nx, ny))

    def get(self, q, name):
        out = np.empty(self.shape(q, name), dtype=np.float64, order="F")
        self._ck(self.lib.pts_batch_get_field(self.h, q, FIELD_ID[name], out.ctypes.data, out.size))
        return out


ASPECT_RATIO_FACTS = (1.0, 0.9, 0.8, 0.7, 0.6, 0.5, 0.4, 0.3, 0.2, 0.1)


def aspect_ratio_instances(facts=ASPECT_RATIO_FACTS, nsubs=(1, 2, 4, 8), resols=(127, 255, 511, 1023, 2047), nt=5,
                           ly=10.0, musi=1e-3):
    """The instances of scripts/runme_Stokes2D_aspect_ratio.jl: FACT x NSUB x RESOL in its
    loop order (Iterators.product: FACT fastest, RESOL slowest), each one run of
    Stokes2D_ve_param.jl."""
    return [dict(ny=ny, nsub=nsub, fact=fact, nt=nt, ly=ly, musi=musi)
            for ny in resols for nsub in nsubs for fact in facts]


class BatchVE(Batch):
    """The visco-elastic aspect-ratio sweep (scripts/Stokes2D_ve_param.jl per instance) in
    one persistent launch (``pts_batch_create_ve``): every instance's nt Maxwell steps,
    with its own check cadence nout = nx and iterMax = 100nx unless `nout` / `iter_max` are
    positive, tolerance eps = 1e-6, CFL 0.87/sqrt(2) (:103-109)."""

    def __init__(self, instances, tile=1, eps=1e-6, CFL=0.87 / math.sqrt(2), Re=5 * math.pi, r=1.0, nout=0,
                 iter_max=0, lib=None):
        self.lib = lib or _abi.load()
        self.instances = []
        for d in instances:
            d = dict(d)
            d.setdefault("nt", 5)
            d.setdefault("ly", 10.0)
            d.setdefault("musi", 1e-3)
            d["nx"] = d["nsub"] * (d["ny"] + 1) - 1
            self.instances.append(d)
        n = len(self.instances)
        arr = (PtsBatchVEInstance * n)()
        for q, d in enumerate(self.instances):
            arr[q] = PtsBatchVEInstance(d["ny"], d["nsub"], d["nt"], 0, d["fact"], d["ly"], d["musi"])
        desc = PtsBatchDesc()
        desc.nout, desc.tile, desc.eps, desc.iter_max = int(nout), tile, eps, float(iter_max)
        desc.r, desc.Re, desc.CFL = r, Re, CFL
        self.desc = desc
        h = ctypes.c_void_p()
        rc = self.lib.pts_batch_create_ve(ctypes.byref(desc), arr, n, ctypes.byref(h))
        if rc != 0:
            raise _abi.PtsError(rc, (self.lib.pts_last_error(None) or b"").decode())
        self.h = h
        self.n = n
        self.tile = tile

    def steps(self, q):
        """PT iterations of each finished Maxwell step of instance q."""
        buf = (ctypes.c_int64 * 64)()
        k = ctypes.c_int32()
        self._ck(self.lib.pts_batch_steps(self.h, q, buf, 64, ctypes.byref(k)))
        return list(buf[: min(k.value, 64)])

    def solve(self, iter_limit=-1, raise_on_nan=True):
        """Run every instance's steps. Result: ittot, err (of each instance's last check),
        converged (its last step reached eps), steps (iterations per step), and the script's
        output line ``nx ny nsub fact ittot nt err`` per instance."""
        from .output import jl

        res = super().solve(iter_limit=iter_limit, raise_on_nan=raise_on_nan)
        res["ittot"] = res.pop("iters")
        res["steps"] = [self.steps(q) for q in range(self.n)]
        res["lines"] = [f"{d['nx']} {d['ny']} {d['nsub']} {jl(d['fact'])} {t} {d['nt']} {jl(e)}"
                        for d, t, e in zip(self.instances, res["ittot"], res["err"])]
        return res

    def shape(self, q, name):
        if name == "txy_o":
            nx, ny = self.instances[q]["nx"], self.instances[q]["ny"]
            return (nx - 1, ny - 1)
        return super().shape(q, name)


def _cache_path():
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "ptstokes", "autotune.json")


def _batch_key(batch):
    cells = sum(d["nx"] * d["ny"] for d in batch.instances)
    classes = sorted({d["nx"] for d in batch.instances})
    form = "ve" if isinstance(batch, BatchVE) else "v"
    return (f"2d|{form}|fp64|n={batch.n}|cells~{2 ** int(math.log2(max(cells, 1)))}|"
            f"nx={','.join(map(str, classes))}")


def autotune(batch, iters=None, use_cache=True):
    """Time each tile shape on `batch` (a Batch or a BatchVE) for a short run from its set-up
    state and keep the fastest; the choice is cached per (form, precision, batch size class)."""
    import torch

    key = _batch_key(batch)
    path = _cache_path()
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            cache = json.load(open(path))
        except Exception:
            cache = {}
    if use_cache and key in cache:
        batch.set_tile(cache[key]["tile"])
        return cache[key]
    if not iters:  # two checks of the instances (a visco-elastic sweep checks every nx iterations)
        nout = batch.desc.nout if batch.desc.nout > 0 else min(d["nx"] for d in batch.instances)
        iters = 2 * nout - 1
    stream = torch.cuda.ExternalStream(batch.stream_handle())
    timings = {}
    for t in range(len(TILE_SHAPES)):
        batch.set_tile(t)
        batch.setup()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        batch.solve(iter_limit=iters)
        b.record(stream)
        b.synchronize()
        timings[t] = a.elapsed_time(b)
    best = min(timings, key=timings.get)
    batch.set_tile(best)
    batch.setup()
    entry = {"tile": best, "shape": TILE_SHAPES[best], "ms": timings, "iters": iters, "when": time.time()}
    if use_cache:
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            cache[key] = entry
            json.dump(cache, open(path, "w"), indent=1)
        except OSError:
            pass
    return entry
