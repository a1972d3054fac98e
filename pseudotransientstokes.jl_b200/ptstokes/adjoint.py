"""Adjoint gradients of the 3D viscous PT solve: ∂J/∂log μ through the C ABI.

The reference has no adjoint. The forward problem is the 3D_V solve (the 3D kernels of
scripts/stokes_3D/Stokes3D_ve_perf.jl without elastic terms) with pure-shear walls; the
objective is a misfit of the vertical velocity on the top interior face plane,
J = ½‖Vz(top) − Vobs‖². ``ViscousAdjoint`` runs the forward solve, the transposed
(adjoint) solve with the source ∂J/∂Vz on that plane, and the pointwise gradient kernel,
all on the device (``pts_gradient_logmu`` in include/ptstokes.h); ``ViscoElasticAdjoint``
does the same for nt Maxwell visco-elastic steps with per-step checkpoints. ``TopVz`` wraps the
same steps as a ``torch.autograd.Function`` of log μ (the viscosity the solver uses, after
any smoothing). ``inclusion_set`` draws the seeded 20-inclusion set, which
``Solver.init_inclusions`` turns into the viscosity field on the device (``viscosity_field``
is the same field computed on the host); ``lognormal_factor`` draws the log-normal
perturbation of the synthetic observations.
"""
import numpy as np

from .solver import Solver


def inclusion_set(count=20, seed=1855, box=(10.0, 10.0, 10.0), radius=(0.3, 0.8), log10_mu=(-4.0, 4.0)):
    """`count` spheres: centres uniform in the box, radii uniform in `radius`, log10 of the
    inclusion viscosity uniform in `log10_mu` (matrix viscosity 1)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        c = [float(rng.uniform(0.0, L)) for L in box]
        out.append(dict(centre=c, radius=float(rng.uniform(*radius)), log10_mu=float(rng.uniform(*log10_mu))))
    return out


def inclusion_array(inclusions, box=(10.0, 10.0, 10.0)):
    """The (count, 5) float64 rows [x, y, z, r2, mus] of pts_init_inclusions: centres in the
    scripts' centred frame (x - lx/2, as Stokes2D_param.jl's Xi, Yi), squared radii and
    viscosities 10**log10_mu."""
    out = np.zeros((len(inclusions), 5), dtype=np.float64)
    for q, inc in enumerate(inclusions):
        c = inc["centre"]
        out[q, 0:3] = [c[0] - 0.5 * box[0], c[1] - 0.5 * box[1], (c[2] if len(c) > 2 else 0.5 * box[2]) - 0.5 * box[2]]
        out[q, 3] = inc["radius"] * inc["radius"]
        out[q, 4] = 10.0 ** inc["log10_mu"]
    return out


def viscosity_field(nx, ny, nz, inclusions, box=(10.0, 10.0, 10.0), mus0=1.0):
    """Cell-centred viscosity (nx, ny, nz), column-major, on the host: the same operations as
    pts_init_inclusions (create_inclusions!, Stokes2D_param.jl:83-99, in 3D): at the cell
    centre x = (ix-1)*dx + 0.5*dx - 0.5*lx, the first inclusion with
    (x-Xi)^2 + (y-Yi)^2 + (z-Zi)^2 < r2 gives 10**log10_mu, else mus0."""
    lx, ly, lz = box
    dx, dy, dz = lx / nx, ly / ny, lz / nz
    rows = inclusion_array(inclusions, box)
    x = (np.arange(nx) * dx + 0.5 * dx) - 0.5 * lx
    y = (np.arange(ny) * dy + 0.5 * dy) - 0.5 * ly
    z = (np.arange(nz) * dz + 0.5 * dz) - 0.5 * lz
    mus = np.full((nx, ny, nz), mus0, dtype=np.float64, order="F")
    # the first hit wins: apply the list backwards, each inclusion overwriting the later ones
    for xi, yi, zi, r2, mu in rows[::-1]:
        ax, ay, az = x - xi, y - yi, z - zi
        rad2 = (ax * ax)[:, None, None] + (ay * ay)[None, :, None]
        rad2 = rad2 + (az * az)[None, None, :]
        mus[rad2 < r2] = mu
    return mus


def lognormal_factor(shape, sigma=0.5, corr=8.0, seed=7):
    """10**(sigma·ξ): ξ is white noise smoothed by a periodic Gaussian of standard deviation
    `corr` cells and rescaled to unit standard deviation."""
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    xi = gaussian_filter(rng.standard_normal(shape), corr, mode="wrap")
    xi = xi / xi.std()
    return np.asfortranarray(10.0 ** (sigma * xi))


def top_plane(vz):
    """Vz on the top interior face plane: the (nx-2, ny-2) interior faces of z-face nz-1."""
    nx, ny, nz1 = vz.shape
    return vz[1:nx - 1, 1:ny - 1, nz1 - 2]


class ViscousAdjoint:
    """Forward solve, adjoint solve and ∂J/∂log μ for J = ½‖Vz(top) − Vobs‖² (or any J whose
    derivative lives on the top Vz plane), on two 3d_v contexts of the same grid."""

    def __init__(self, nx, ny, nz, ebg=1.0, lib=None, **kw):
        self.nx, self.ny, self.nz, self.ebg = nx, ny, nz, ebg
        self.fwd = Solver("3d_v", nx, ny, nz, lib=lib, **kw)
        self.adj = Solver("3d_v", nx, ny, nz, lib=lib, adjoint=1, **kw)
        self.mus = None

    def close(self):
        self.fwd.close()
        self.adj.close()

    def set_viscosity(self, mus, nsmooth=10):
        """Mus = mus smoothed nsmooth times on the device (smooth!, as the scripts do). The
        gradient is with respect to the log of the smoothed field (``self.mus``)."""
        f = self.fwd
        f.init_inclusion(1.0, 1.0, 0.0, self.ebg)
        f.set("Mus", mus)
        if nsmooth:
            f.smooth(nsmooth, 1.0)
        self.mus = f.get("Mus")
        return self

    def set_inclusions(self, inclusions, nsmooth=10, box=(10.0, 10.0, 10.0)):
        """Mus built on the device from a list of spheres (``inclusion_set`` dicts; the first
        sphere a cell centre is inside gives its viscosity, else 1), then smoothed nsmooth
        times there: no host-built field crosses to the device. ``self.mus`` is a host copy."""
        import torch

        f = self.fwd
        f.init_inclusions(inclusion_array(inclusions, box), mus0=1.0, ebg=self.ebg)
        if nsmooth:
            f.smooth(nsmooth, 1.0)
        self.mus = f.get("Mus")
        t = torch.empty(self.mus.size, dtype=torch.float64, device="cuda")
        f.get_device("Mus", t.data_ptr(), t.numel())
        self._mus_dev, self._mus_src = t, self.mus
        return self

    def _load_mus(self, s):
        """Mus of context s = the current viscosity: a device-to-device copy while ``self.mus``
        is the field the device copy was made from, else an upload of ``self.mus``."""
        import torch

        if getattr(self, "_mus_src", None) is not self.mus:
            self._mus_dev = torch.from_numpy(np.ascontiguousarray(self.mus.ravel(order="F"))).to("cuda")
            self._mus_src = self.mus
        torch.cuda.synchronize()
        s.set_device("Mus", self._mus_dev.data_ptr(), self._mus_dev.numel())

    def forward(self):
        """The forward PT solve from the pure-shear initial state (walls and ICs, Mus, the
        local-max viscosity and the iteration parameters); returns its outcome (pts_solve)."""
        f = self.fwd
        f.init_inclusion(1.0, 1.0, 0.0, self.ebg)
        self._load_mus(f)
        f.compute_maxloc()
        f.compute_iter_params()
        return f.solve()

    def top_vz(self):
        return top_plane(self.fwd.get("Vz")).copy(order="F")

    def adjoint(self, dJ_dtop):
        """The transposed solve with the momentum source dJ/dVz on the top interior plane."""
        a = self.adj
        a.init_inclusion(1.0, 1.0, 0.0, 0.0)  # every field zero; walls and ghosts zero
        self._load_mus(a)
        a.compute_maxloc()
        a.compute_iter_params()
        Fz = np.zeros(a.shape("Fz"), order="F")
        Fz[:, :, -1] = dJ_dtop
        a.set("Fz", Fz)
        return a.solve()

    def gradient(self):
        """∂J/∂log μ per cell (nx, ny, nz) from the last forward and adjoint solves."""
        self.fwd.gradient_logmu(self.adj)
        return self.fwd.get("grad")

    def misfit_gradient(self, vobs):
        """J and ∂J/∂log μ for J = ½‖Vz(top) − Vobs‖² at the current viscosity."""
        fo = self.forward()
        r = self.top_vz() - vobs
        J = 0.5 * float(np.sum(r * r))
        ao = self.adjoint(r)
        return J, self.gradient(), fo, ao


class ViscoElasticAdjoint:
    """∂J/∂log μ of J = ½‖Vz(top, last step) − Vobs‖² for nt Maxwell visco-elastic time steps
    (the 3D_VE_PERF kernels, each step converged to eps), on two contexts of the same grid.

    The forward time loop stores each step's converged stresses (a per-step checkpoint, on
    the host). The adjoint is the same time loop on an adjoint-mode context, run backwards:
    assign_τ! (τ_o ← τ) between steps as forward, the source ∂J/∂Vz only in the first
    adjoint step; after adjoint step s the forward context's stresses are restored from
    checkpoint nt-1-s and the step's gradient term is accumulated (pts_gradient_logmu_add)."""

    TAU = ("txx", "tyy", "tzz", "txy", "txz", "tyz")

    def __init__(self, nx, ny, nz, nt=5, ebg=1.0, lib=None, **kw):
        kw.setdefault("nout", 200)
        kw.setdefault("iter_max", 2e5)
        kw.setdefault("eps", 1e-8)
        self.nx, self.ny, self.nz, self.nt, self.ebg = nx, ny, nz, nt, ebg
        self.fwd = Solver("3d_ve_perf", nx, ny, nz, lib=lib, **kw)
        self.adj = Solver("3d_ve_perf", nx, ny, nz, lib=lib, adjoint=1, **kw)
        self.mus = None
        self.checkpoints = []

    def close(self):
        self.fwd.close()
        self.adj.close()

    set_viscosity = ViscousAdjoint.set_viscosity
    set_inclusions = ViscousAdjoint.set_inclusions
    top_vz = ViscousAdjoint.top_vz

    _load_mus = ViscousAdjoint._load_mus

    def _prepare(self, s, ebg):
        s.init_inclusion(1.0, 1.0, 0.0, ebg)
        self._load_mus(s)
        s.compute_maxloc()
        s.compute_iter_params()

    def forward(self):
        """nt physical steps from the pure-shear initial state; returns the per-step outcomes."""
        f = self.fwd
        self._prepare(f, self.ebg)
        self.checkpoints, out = [], []
        for _ in range(self.nt):
            f.assign_tau()
            out.append(f.solve())
            self.checkpoints.append([f.get(n) for n in self.TAU])
        return out

    def adjoint(self, dJ_dtop):
        """The backward adjoint time loop with the gradient accumulated step by step."""
        a, f = self.adj, self.fwd
        self._prepare(a, 0.0)  # every field zero
        Fz = np.zeros(a.shape("Fz"), order="F")
        Fz[:, :, -1] = dJ_dtop
        a.set("Fz", Fz)
        out = []
        for s in range(self.nt):
            a.assign_tau()
            out.append(a.solve())
            for n, t in zip(self.TAU, self.checkpoints[self.nt - 1 - s]):
                f.set(n, t)
            f.gradient_logmu(a, add=s > 0)
            if s == 0:
                a.set("Fz", np.zeros_like(Fz))
        return out

    def gradient(self):
        return self.fwd.get("grad")

    def misfit_gradient(self, vobs):
        """J and ∂J/∂log μ for J = ½‖Vz(top) − Vobs‖² after the last step."""
        fo = self.forward()
        r = self.top_vz() - vobs
        J = 0.5 * float(np.sum(r * r))
        ao = self.adjoint(r)
        return J, self.gradient(), fo, ao


def _torch_function():
    import torch

    class TopVz(torch.autograd.Function):
        """Vz on the top interior plane as a differentiable function of log μ (float64,
        shape (nx, ny, nz), the viscosity the solver uses). Forward: one PT solve; backward:
        the transposed solve with the incoming gradient as source, then ∂/∂log μ."""

        @staticmethod
        def forward(ctx, logmu, problem):
            mus = torch.exp(logmu.detach()).cpu().numpy()
            problem.set_viscosity(np.asfortranarray(mus), nsmooth=0)
            problem.forward()
            ctx.problem = problem
            return torch.from_numpy(problem.top_vz()).to(logmu.device)

        @staticmethod
        def backward(ctx, g):
            p = ctx.problem
            p.adjoint(np.asfortranarray(g.detach().cpu().numpy()))
            return torch.from_numpy(p.gradient()).to(g.device), None

    return TopVz


def top_vz(logmu, problem):
    """Differentiable Vz(top) of log μ (see ``TopVz``)."""
    return _torch_function().apply(logmu, problem)
