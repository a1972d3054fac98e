"""The z-slab decomposition (ptstokes.multi, the ImplicitGlobalGrid part of
Stokes3D_ve_multixpu.jl) on two gloo ranks on the CPU. Each rank's local solver is the
oracle's restatement of the script's kernels on its slab (global z coordinates in the initial
conditions, global dz), and the halo planes move through torch.distributed point-to-point
calls: after the set-up and 30 PT iterations, the slabs glued back together equal a
single-domain run of the global grid bit for bit, and the reduced check counts the overlap
planes on both ranks, as the reference's norm_g does."""
import math
import os
import socket
import sys

import numpy as np

from conftest import ROOT

NX, NY, NZ_G, ITERS = 17, 15, 22, 30
FIELDS = ("Pt", "Vx", "Vy", "Vz", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Mus", "Must")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def oracle_slab(nx, ny, slabs, exchange_fn):
    """The oracle's Stokes3D_ve_multixpu.jl case on one slab: dz = lz/nz_g, the initial
    conditions at the global z coordinate z_g (ImplicitGlobalGrid: (coords*(nz-2)+iz-1)*dz + z0),
    and update_halo! of Mus after each smoothing sweep and of Musτ after the local maximum."""
    from oracle import scripts as S
    from oracle.binding import arr

    class Slab(S.VE3D):
        _allocating = False

        def setup(self):
            self._allocating = True
            super().setup()  # allocations only: its dz and ICs are replaced below
            self._allocating = False
            nz, dx, dy, lx, ly, lz = self.nz, self.dx, self.dy, self.lx, self.ly, self.lz
            self.dz = lz / slabs.nz_global
            self._dz = 1.0 / self.dz
            self.Vpdt = min(self.dx, self.dy, self.dz) * self.CFL
            dz = self.dz
            ix = np.arange(1, nx + 2, dtype=np.float64)
            iy = np.arange(1, ny + 1, dtype=np.float64)
            izg = np.arange(1, nz + 2, dtype=np.float64) + slabs.zoff  # global plane index + 1
            xv = ((ix - 1) * dx + (-0.5 * dx)) + 0.5 * dx - 0.5 * lx
            zv = ((izg - 1) * dz + (-0.5 * dz)) + 0.5 * dz - 0.5 * lz
            X = ((ix[:nx] - 1) * dx + 0.0) + 0.5 * dx - 0.5 * lx
            Y = ((iy - 1) * dy + 0.0) + 0.5 * dy - 0.5 * ly
            Z = ((izg[:nz] - 1) * dz + 0.0) + 0.5 * dz - 0.5 * lz
            Rad2 = (X[:, None, None] ** 2 + Y[None, :, None] ** 2) + Z[None, None, :] ** 2
            self.f["Vx"] = np.asfortranarray(np.broadcast_to((-self.ebg * xv)[:, None, None], (nx + 1, ny, nz)))
            self.f["Vz"] = np.asfortranarray(np.broadcast_to((self.ebg * zv)[None, None, :], (nx, ny, nz + 1)))
            for k in ("Pt", "divV", "txx", "tyy", "tzz", "txy", "txz", "tyz", "dVx", "dVy", "dVz"):
                self.f[k][...] = 0.0
            self.f["Vy"][...] = 0.0
            Mus = self.mus0 * np.ones((nx, ny, nz), order="F")
            Mus[Rad2 < 1.0] = self.musi
            self.init_viscosity(Mus)
            return self

        def init_viscosity(self, Mus):
            if self._allocating:
                return
            L = self.L
            Mus = np.asfortranarray(Mus, dtype=np.float64)
            Mus2 = self.f["Mus2"]
            Mus2[...] = Mus
            for _ in range(10):
                L.ora3_smooth(arr(Mus2), arr(Mus), 1.0)
                Mus, Mus2 = Mus2, Mus
                self.f["Mus"], self.f["Mus2"] = Mus, Mus2
                exchange_fn(self, ("Mus",))
            Must = self.f["Must"]
            Must[...] = Mus
            L.ora3_maxloc(arr(Must), arr(Mus))
            L.ora3_bc_x(arr(Must))
            L.ora3_bc_y(arr(Must))
            L.ora3_bc_z(arr(Must))
            exchange_fn(self, ("Must",))
            self.iter_params()

    return Slab(nx, ny, slabs.nz)


class _HostPlanes:
    """get_plane/set_plane of the oracle's numpy fields for ptstokes.multi.exchange."""

    def __init__(self, case):
        self.c = case

    def shape(self, name):
        return self.c.f[name].shape

    def plane_like(self, name):
        import torch

        e = self.shape(name)
        return torch.empty(e[0] * e[1], dtype=torch.float64)

    def get_plane(self, name, k):
        import torch

        return torch.from_numpy(np.ascontiguousarray(self.c.f[name][:, :, k].ravel(order="F")))

    def set_plane(self, name, k, buf):
        e = self.shape(name)
        self.c.f[name][:, :, k] = buf.numpy().reshape(e[0], e[1], order="F")


def _rank_main(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    for p in (ROOT, os.path.join(ROOT, "pseudotransientstokes.jl_b200")):
        sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    from oracle.binding import stats
    from ptstokes.multi import Slabs, exchange, global_check

    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=60))
    try:
        slabs = Slabs(NZ_G, 2, rank)

        def ex(case, names):
            exchange(_HostPlanes(case), names, slabs, dist)

        c = oracle_slab(NX, NY, slabs, ex)
        c.setup()
        c.assign_tau()
        for _ in range(ITERS):
            c.iteration()
            ex(c, ("Vx", "Vy", "Vz"))
        c.check()  # Rx, Ry, Rz of the current fields
        part = [stats(c.f[k])[0] for k in ("Rx", "Ry", "Rz", "divV")]
        _, vmin, vmax = stats(c.f["Vx"])
        _, pmin, pmax = stats(c.f["Pt"])
        err, norms = global_check(part + [vmin, vmax, pmin, pmax], slabs, NX, NY, c.lx, dist)
        out.put((rank, {k: c.f[k] for k in FIELDS}, err, norms, part + [vmin, vmax, pmin, pmax]))
    finally:
        dist.destroy_process_group()


def test_two_slabs_equal_the_global_grid():
    import torch.multiprocessing as mp

    from oracle import scripts as S
    from oracle.binding import stats
    from ptstokes.multi import Slabs, assemble

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slabs = [Slabs(NZ_G, 2, r) for r in range(2)]

    g = S.make("3d_ve", NX, NY, NZ_G)
    g.setup()
    g.assign_tau()
    for _ in range(ITERS):
        g.iteration()
    for k in FIELDS:
        glued = assemble([res[0][1][k], res[1][1][k]], slabs)
        assert glued.shape == g.f[k].shape, k
        assert np.array_equal(glued, g.f[k]), k
    # the overlap planes agree on both ranks
    for k in ("Vx", "Vy", "Vz", "Pt", "Mus"):
        a, b = res[0][1][k], res[1][1][k]
        ol = slabs[1].overlap(b.shape[2])
        assert np.array_equal(a[:, :, a.shape[2] - ol:], b[:, :, :ol]), k
    # the reduced check: both ranks get the same err, from sums that count the overlap twice
    assert res[0][2] == res[1][2] and math.isfinite(res[0][2])
    g.check()
    sums = [stats(g.f[k])[0] for k in ("Rx", "Ry", "Rz", "divV")]
    tot = [a + b for a, b in zip(res[0][4][:4], res[1][4][:4])]
    assert all(t >= s * (1 - 1e-12) for t, s in zip(tot, sums))
    err_g, _ = g.check()
    assert abs(res[0][2] - err_g) <= 0.2 * err_g


def test_slab_geometry():
    from ptstokes.multi import Slabs

    s = Slabs(66, 4, 2)
    assert (s.nz, s.zoff, s.down, s.up) == (18, 32, 1, 3)
    assert s.overlap(18) == 2 and s.overlap(19) == 3 and s.overlap(16) == 0
    one = Slabs(34, 1, 0)
    assert one.global_lengths(17, 15) == (16 * 13 * 32, 15 * 14 * 32, 15 * 13 * 33, 17 * 15 * 34)
    import pytest

    with pytest.raises(ValueError):
        Slabs(65, 4, 0)
