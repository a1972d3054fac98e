"""Multi-GPU z-slab decomposition: the ImplicitGlobalGrid part of
scripts/stokes_3D/Stokes3D_ve_multixpu.jl, along z, over torch.distributed.

The reference decomposes the global grid over MPI ranks with ImplicitGlobalGrid
(init_global_grid, :138): each rank holds nx x ny x nz cells whose outer planes overlap the
neighbours' by two, so nz_g = P*(nz-2) + 2 along a line of P ranks. After every PT iteration
the V update is followed by update_halo!(Vx, Vy, Vz) (:238), and during set-up by
update_halo!(Mus) after each smoothing sweep and update_halo!(Musτ) after the local maximum
(:182-195). The convergence check reduces over ranks: norm_g, minimum_g, maximum_g, with the
global lengths len_*_g (:192-195, :243-248).

Here each rank is one process with one GPU context holding its slab (``SlabSolver``), the
halo planes move between neighbours with torch.distributed point-to-point calls (NCCL on
GPUs, gloo on the CPU), and the check's sums, minima and maxima are all-reduced. A halo
exchange (``exchange``) works on any local object with get_plane/set_plane/plane_like, so
the same code drives the CPU oracle in the tests.

Overlap of a field (ImplicitGlobalGrid's ol(dim, A) = 2 + size(A, dim) - nz): 2 for cell
arrays (Vx, Vy, Mus, Musτ: nz planes), 3 for Vz (nz+1 z-faces). The last ol planes of rank r
are the first ol planes of rank r+1, and with a halo of one plane: rank r's last plane takes
rank r+1's plane ol-1, and rank r+1's first plane takes rank r's plane n-ol (0-based, n the
field's local z-extent).
"""
import ctypes
import math

import numpy as np

from .solver import Solver


class Slabs:
    """Geometry of a line of `size` ranks along z over a global grid of nz_global cells."""

    def __init__(self, nz_global, size, rank):
        if size < 1 or not 0 <= rank < size:
            raise ValueError("rank out of range")
        if (nz_global - 2) % size:
            raise ValueError(f"nz_global - 2 = {nz_global - 2} is not a multiple of {size} ranks")
        self.size, self.rank = size, rank
        self.nz_global = nz_global
        self.nz = (nz_global - 2) // size + 2        # init_global_grid: nz_g = P*(nz-2) + 2
        self.zoff = rank * (self.nz - 2)             # z_g: coords*(nz - overlap)
        self.down = rank - 1 if rank > 0 else None
        self.up = rank + 1 if rank < size - 1 else None

    def overlap(self, n):
        """ol(dim, A) of a field with n local z-planes."""
        return 2 + (n - self.nz)

    def global_lengths(self, nx, ny):
        """len_Rx_g, len_Ry_g, len_Rz_g, len_∇V_g of Stokes3D_ve_multixpu.jl:192-195 for dims
        (1, 1, size) (overlap planes are counted on both ranks, as the reference does)."""
        P, nz = self.size, self.nz
        return ((nx - 3 + 2) * (ny - 4 + 2) * ((nz - 4) * P + 2),
                (nx - 4 + 2) * (ny - 3 + 2) * ((nz - 4) * P + 2),
                (nx - 4 + 2) * (ny - 4 + 2) * ((nz - 3) * P + 2),
                (nx - 2 + 2) * (ny - 2 + 2) * ((nz - 2) * P + 2))


def exchange(local, names, slabs, dist, group=None):
    """update_halo!(names...) along z between neighbour ranks (point-to-point; every rank makes
    the same calls in the same order). `local` provides shape(name), get_plane(name, k),
    set_plane(name, k, plane) and plane buffers that `dist` can send."""
    if slabs.size == 1:
        return
    ops, recvs = [], []
    for name in names:
        n = local.shape(name)[2]
        ol = slabs.overlap(n)
        if slabs.up is not None:
            ops.append(dist.P2POp(dist.isend, local.get_plane(name, n - ol), slabs.up, group))
            buf = local.plane_like(name)
            ops.append(dist.P2POp(dist.irecv, buf, slabs.up, group))
            recvs.append((name, n - 1, buf))
        if slabs.down is not None:
            ops.append(dist.P2POp(dist.isend, local.get_plane(name, ol - 1), slabs.down, group))
            buf = local.plane_like(name)
            ops.append(dist.P2POp(dist.irecv, buf, slabs.down, group))
            recvs.append((name, 0, buf))
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    if recvs and recvs[0][2].is_cuda:  # the received planes are copied on the context's stream
        import torch

        torch.cuda.synchronize()
    for name, k, buf in recvs:
        local.set_plane(name, k, buf)


def exchange_local(locals_, slabs_list, names):
    """update_halo!(names...) between slabs held by one process (several contexts, on one GPU
    or several): the planes of ``exchange`` move by device-to-device copies. The planes read
    (ol-1 and n-ol) are never halo planes, so the order of the copies does not matter."""
    for r in range(len(locals_) - 1):
        lo, up = locals_[r], locals_[r + 1]
        for name in names:
            n = lo.shape(name)[2]
            ol = slabs_list[r].overlap(n)
            a, b = lo.get_plane(name, n - ol), up.get_plane(name, ol - 1)
            up.set_plane(name, 0, a)
            lo.set_plane(name, n - 1, b)


def combine_partials(parts):
    """The rank reduction of check partials done in one process."""
    return ([sum(p[q] for p in parts) for q in range(4)] +
            [min(p[4] for p in parts), max(p[5] for p in parts), min(p[6] for p in parts), max(p[7] for p in parts)])


def global_check(partials, slabs, nx, ny, lx, dist, group=None, device="cpu"):
    """err and the four norms from each rank's {Σ Rx², Σ Ry², Σ Rz², Σ ∇V², min Vx, max Vx,
    min Pt, max Pt} (Stokes3D_ve_multixpu.jl:243-248: norm_g, minimum_g, maximum_g)."""
    import torch

    p = list(partials)
    if slabs.size > 1 and dist is not None:
        s = torch.tensor(p[:4], dtype=torch.float64, device=device)
        lo = torch.tensor([p[4], p[6]], dtype=torch.float64, device=device)
        hi = torch.tensor([p[5], p[7]], dtype=torch.float64, device=device)
        dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(lo, op=dist.ReduceOp.MIN, group=group)
        dist.all_reduce(hi, op=dist.ReduceOp.MAX, group=group)
        p = s.tolist() + [lo[0].item(), hi[0].item(), lo[1].item(), hi[1].item()]
    lRx, lRy, lRz, lDiv = slabs.global_lengths(nx, ny)
    dP, dV = p[7] - p[6], p[5] - p[4]
    norms = [math.sqrt(p[0]) / dP * lx / math.sqrt(lRx), math.sqrt(p[1]) / dP * lx / math.sqrt(lRy),
             math.sqrt(p[2]) / dP * lx / math.sqrt(lRz), math.sqrt(p[3]) / dV * lx / math.sqrt(lDiv)]
    err = float("nan") if any(math.isnan(v) for v in norms) else max(norms)
    return err, norms


B_WIDTH_Z = 4  # the z component of b_width = (8, 4, 4) (Stokes3D_ve_multixpu.jl:136)


def _overlap_begin(s, side, bz):
    """One PT iteration of context `s` as @hide_communication b_width (Stokes3D_ve_multixpu.jl:
    230-239): compute_P! + compute_τ!, then compute_V! + bc on the bz face planes at each end of
    the slab on the context's stream and on the inner planes on the stream `side` (after
    compute_τ!). The halo planes that update_halo! reads and writes lie in the end regions, so
    the exchange can start once the context's stream is done while the inner planes are still
    being updated. Returns (context stream, event of the inner update) for _overlap_end."""
    import torch

    cs = torch.cuda.ExternalStream(s.stream_handle())
    s.compute_Pt_tau()
    nf = s.nz + 1  # face planes of Vz, the z-extent of the update
    lib, ctx = s.lib, s.ctx
    if nf > 2 * bz:
        ready = torch.cuda.Event()
        ready.record(cs)
        side.wait_event(ready)
        s._ck(lib.pts_compute_V_bc_planes(ctx, bz, nf - bz, ctypes.c_void_p(side.cuda_stream)))
        s._ck(lib.pts_compute_V_bc_planes(ctx, 0, bz, None))
        s._ck(lib.pts_compute_V_bc_planes(ctx, nf - bz, nf, None))
        done = torch.cuda.Event()
        done.record(side)
        return cs, done
    s._ck(lib.pts_compute_V_bc_planes(ctx, 0, nf, None))
    return cs, None


def _overlap_end(cs, done):
    """The context's stream waits for the inner planes' update before its next work."""
    if done is not None:
        cs.wait_event(done)


class _DevicePlanes:
    """get_plane/set_plane of a GPU context's fields through dense device buffers."""

    def __init__(self, s):
        self.s = s

    def shape(self, name):
        return self.s.shape(name)

    def plane_like(self, name):
        import torch

        e = self.shape(name)
        return torch.empty(e[0] * e[1], dtype=torch.float64, device="cuda")

    def get_plane(self, name, k):
        from ._abi import FIELD_ID

        buf = self.plane_like(name)
        self.s._ck(self.s.lib.pts_get_plane_device(self.s.ctx, FIELD_ID[name], k, buf.data_ptr(), buf.numel()))
        return buf

    def set_plane(self, name, k, buf):
        from ._abi import FIELD_ID

        self.s._ck(self.s.lib.pts_set_plane_device(self.s.ctx, FIELD_ID[name], k, buf.data_ptr(), buf.numel()))


class SlabSolver:
    """One rank's slab of a 3D problem decomposed along z (``Stokes3D_ve_multixpu.jl`` with
    dims = (1, 1, P)): a local GPU context of nx x ny x nz cells, nz = (nz_g-2)/P + 2, whose
    initial conditions use the global z coordinate, with halo exchanges and a reduced check.
    ``dist`` is torch.distributed with an initialised process group (NCCL for GPUs)."""

    def __init__(self, variant, nx, ny, nz_global, dist, group=None, lib=None, overlap=False, b_width=B_WIDTH_Z,
                 **kw):
        """With `overlap`, each iteration hides its halo exchange behind the update of the inner
        planes, as @hide_communication b_width does (b_width: face planes at each slab end)."""
        self.dist, self.group = dist, group
        self.overlap, self.b_width = overlap, int(b_width)
        size = dist.get_world_size(group) if dist is not None else 1
        rank = dist.get_rank(group) if dist is not None else 0
        self.slabs = Slabs(nz_global, size, rank)
        self.nx, self.ny = nx, ny
        self.s = Solver(variant, nx, ny, self.slabs.nz, lib=lib, **kw)
        self.s._ck(self.s.lib.pts_set_decomposition(self.s.ctx, self.slabs.zoff, nz_global))
        self.planes = _DevicePlanes(self.s)
        self.lx = self.s.p["lx"]
        if overlap:
            import torch

            self.side = torch.cuda.Stream()

    def close(self):
        self.s.close()

    def halo(self, *names):
        self.s.sync()
        exchange(self.planes, names, self.slabs, self.dist, self.group)

    def setup_inclusion(self, musi=1e-3, radius2=1.0, ebg=1.0, nsmooth=10):
        """The script's set-up with its halo updates (Stokes3D_ve_multixpu.jl:173-192)."""
        s = self.s
        s.init_inclusion(s.p["mus0"], musi, radius2, ebg)
        for _ in range(nsmooth):
            s.smooth(1, 1.0)
            self.halo("Mus")
        s.compute_maxloc()
        self.halo("Must")
        s.compute_iter_params()
        return self

    def assign_tau(self):
        self.s.assign_tau()

    def iteration(self):
        """compute_P!, compute_τ!, compute_dV!, compute_V! + bc, then update_halo!(Vx, Vy, Vz);
        with overlap, the exchange runs while the inner planes are updated."""
        if self.overlap:
            cs, done = _overlap_begin(self.s, self.side, self.b_width)
            self.halo("Vx", "Vy", "Vz")
            _overlap_end(cs, done)
            return
        self.s.iterate(1)
        self.halo("Vx", "Vy", "Vz")

    def check(self):
        out = (__import__("ctypes").c_double * 8)()
        self.s._ck(self.s.lib.pts_check_partials(self.s.ctx, out))
        dev = "cuda" if self.dist is not None and self.dist.get_backend(self.group) == "nccl" else "cpu"
        return global_check(list(out), self.slabs, self.nx, self.ny, self.lx, self.dist, self.group, dev)

    def solve(self, eps=None, iter_max=None, nout=None):
        """One physical step's PT loop (`while err > ε && iter <= iterMax`, check every nout)."""
        p = self.s.p
        eps = p["eps"] if eps is None else eps
        iter_max = p["iter_max"] if iter_max is None else iter_max
        nout = int(p["nout"] if nout is None else nout)
        err, it = 2 * eps, 0
        norms = None
        while err > eps and it <= iter_max:
            self.iteration()
            it += 1
            if it % nout == 0:
                err, norms = self.check()
                if math.isnan(err):
                    raise FloatingPointError("NaN in the residual check")
        return dict(iters=it, err=err, norms=norms, converged=not err > eps)

    def run(self, nt=None, **kw):
        """The time loop: assign_τ! and a converged PT loop per physical step."""
        nt = self.s.p["nt"] if nt is None else nt
        out = []
        for _ in range(nt):
            self.assign_tau()
            out.append(self.solve(**kw))
        return out

    def get_local(self, name):
        return self.s.get(name)


class SlabGroup:
    """All slabs of a z-decomposition driven from one process: one context per slab (each on
    the device current when it is created), halo planes moved by device copies
    (``exchange_local``) and the check reduced on the host. The same numerics as P ranks of
    ``SlabSolver``; for several GPUs in one process, or to run a decomposition on one GPU."""

    def __init__(self, variant, nx, ny, nz_global, nslabs, devices=None, lib=None, overlap=False, b_width=B_WIDTH_Z,
                 **kw):
        import torch

        self.overlap, self.b_width = overlap, int(b_width)
        self.sides = []
        self.slabs = [Slabs(nz_global, nslabs, r) for r in range(nslabs)]
        self.nx, self.ny = nx, ny
        self.solvers, self.planes = [], []
        for r, sl in enumerate(self.slabs):
            if devices is not None:
                torch.cuda.set_device(devices[r])
            s = Solver(variant, nx, ny, sl.nz, lib=lib, **kw)
            s._ck(s.lib.pts_set_decomposition(s.ctx, sl.zoff, nz_global))
            self.solvers.append(s)
            self.planes.append(_DevicePlanes(s))
            if overlap:
                self.sides.append(torch.cuda.Stream())
        self.lx = self.solvers[0].p["lx"]

    def close(self):
        for s in self.solvers:
            s.close()

    def halo(self, *names):
        for s in self.solvers:
            s.sync()
        exchange_local(self.planes, self.slabs, names)

    def setup_inclusion(self, musi=1e-3, radius2=1.0, ebg=1.0, nsmooth=10):
        for s in self.solvers:
            s.init_inclusion(s.p["mus0"], musi, radius2, ebg)
        for _ in range(nsmooth):
            for s in self.solvers:
                s.smooth(1, 1.0)
            self.halo("Mus")
        for s in self.solvers:
            s.compute_maxloc()
        self.halo("Must")
        for s in self.solvers:
            s.compute_iter_params()
        return self

    def assign_tau(self):
        for s in self.solvers:
            s.assign_tau()

    def iteration(self):
        if self.overlap:
            pend = [_overlap_begin(s, side, self.b_width) for s, side in zip(self.solvers, self.sides)]
            self.halo("Vx", "Vy", "Vz")
            for cs, done in pend:
                _overlap_end(cs, done)
            return
        for s in self.solvers:
            s.iterate(1)
        self.halo("Vx", "Vy", "Vz")

    def check(self):
        import ctypes

        parts = []
        for s in self.solvers:
            out = (ctypes.c_double * 8)()
            s._ck(s.lib.pts_check_partials(s.ctx, out))
            parts.append(list(out))
        return global_check(combine_partials(parts), self.slabs[0], self.nx, self.ny, self.lx, None)

    solve = SlabSolver.solve
    run = SlabSolver.run

    @property
    def s(self):
        return self.solvers[0]

    def get(self, name):
        """A field of the whole grid, glued from the slabs."""
        return assemble([s.get(name) for s in self.solvers], self.slabs)


def local_ranges(slabs, nz_field):
    """The global z-planes [g0, g0 + n) of a field with nz_field local planes on this rank."""
    return slabs.zoff, slabs.zoff + nz_field


def assemble(parts, slabs_list, axis=2):
    """Glue local fields of all ranks back into a global array (overlap planes taken from the
    lower rank); for tests and output."""
    out = [parts[0]]
    for r in range(1, len(parts)):
        ol = slabs_list[r].overlap(parts[r].shape[axis])
        out.append(np.take(parts[r], range(ol, parts[r].shape[axis]), axis=axis))
    return np.concatenate(out, axis=axis)
