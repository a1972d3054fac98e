"""Oracle drivers: CPU restatements of the reference scripts' solver functions.

Each ``Case`` subclass mirrors one script of PTsolvers/PseudoTransientStokes.jl:

  ``V2D``        scripts/Stokes2D.jl:72-169             (2D viscous, 4 role kernels)
  ``VE2D``       scripts/Stokes2D_ve.jl:87-206          (2D Maxwell VE, 4 role kernels)
  ``VE2DPerf``   scripts/Stokes2D_ve_perf.jl:80-197     (2D VE, fused explicit-index kernels)
  ``VE3D``       scripts/stokes_3D/Stokes3D_ve_multixpu.jl:118-295 (3D VE, 1 rank)
  ``VE3DPerf``   scripts/stokes_3D/Stokes3D_ve_perf.jl:116-255     (3D VE, fused kernels)
  ``VE2DDamp``   scripts/previous_damp/Stokes2D_ve0.jl:82-204 (2D VE, damped scheme)
  ``V2DDamp``    scripts/previous_damp/Stokes2D0.jl:72-173    (2D viscous, damped scheme)
  ``V3DDamp``    scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl:96-248 (3D viscous, damped, 1 rank)
  ``V3D``        3D viscous: no reference script; the 3D perf kernels with the elastic
                 terms removed and the viscous iteration parameters of Stokes2D.jl:27-31.

Arrays are Float64 column-major numpy arrays with the reference's own extents, so the
oracle state can be compared field by field with the CUDA path (test infrastructure only).
"""
import math

import numpy as np

from .binding import lib, arr, stats

PI = math.pi


def linrange(a, b, n):
    """Julia ``LinRange(a, b, n)`` element values: (1-t)*a + t*b with t = (i-1)/(n-1)."""
    out = np.empty(n)
    d = n - 1
    for j in range(n):
        t = j / d if d > 0 else 0.0
        out[j] = (1 - t) * a + t * b
    return out


def zeros(*shape):
    return np.zeros(shape, dtype=np.float64, order="F")


class Case:
    """Common driver state. Subclasses set the per-script physics, numerics and kernels."""

    ndim = 2
    elastic = True
    # numerics defaults (overridable through keyword arguments)
    defaults = {}

    def __init__(self, nx, ny, nz=None, **kw):
        self.nx, self.ny, self.nz = nx, ny, nz
        p = dict(lx=10.0, ly=10.0, lz=10.0, xi=1.0, mus0=1.0, musi=1e-3, G=1.0, ebg=1.0)
        p.update(self.defaults)
        p.update(kw)
        self.p = p
        for k, v in p.items():
            setattr(self, k, v)
        self.dt = self.mus0 / (self.G * self.xi)
        self.L = lib()
        self.f = {}
        self.iters = []
        self.err_hist = []

    # ---------------------------------------------------------------- helpers
    def A(self, name):
        return arr(self.f[name])

    def alloc(self, **shapes):
        for k, s in shapes.items():
            self.f[k] = zeros(*s)

    # ---------------------------------------------------------------- driver
    def run(self, nt=None, iter_max=None, nout=None, eps=None):
        """The reference's time loop + PT loop (e.g. Stokes3D_ve_perf.jl:192-226)."""
        nt = self.nt if nt is None else nt
        iter_max = self.iterMax if iter_max is None else iter_max
        nout = self.nout if nout is None else nout
        eps = self.eps if eps is None else eps
        self.ittot = 0
        for it in range(1, nt + 1):
            err = 2 * eps
            it_ = 0
            if self.elastic:
                self.assign_tau()
            while err > eps and it_ <= iter_max:
                self.iteration()
                it_ += 1
                if it_ % nout == 0:
                    err, norms = self.check()
                    self.err_hist.append((it, it_, err, norms))
                    if math.isnan(err):
                        raise FloatingPointError("NaN")
            self.iters.append(it_)
            self.ittot += it_
        return self

    def norm_err(self, names_R, name_div, len_over=None):
        """err = max(norm_R..., norm_∇V) as in Stokes3D_ve_perf.jl:211-218."""
        _, vmin, vmax = stats(self.f["Vx"])
        _, pmin, pmax = stats(self.f["Pt"])
        norms = []
        for n in names_R:
            s, _, _ = stats(self.f[n])
            norms.append(math.sqrt(s) / (pmax - pmin) * self.lx / math.sqrt(self.f[n].size))
        s, _, _ = stats(self.f[name_div])
        norms.append(math.sqrt(s) / (vmax - vmin) * self.lx / math.sqrt(self.f[name_div].size))
        return max(norms), norms


class _Case2D(Case):
    ndim = 2

    def setup(self):
        """Allocations, initial conditions and iteration parameters (Stokes2D.jl:87-125)."""
        nx, ny, L = self.nx, self.ny, self.L
        self.dx, self.dy = self.lx / nx, self.ly / ny
        self._dx, self._dy = 1.0 / self.dx, 1.0 / self.dy
        self.max_lxy = max(self.lx, self.ly)
        self.Vpdt = min(self.dx, self.dy) * self.CFL
        self.xc = linrange(self.dx / 2, self.lx - self.dx / 2, nx)
        self.yc = linrange(self.dy / 2, self.ly - self.dy / 2, ny)
        self.alloc(Pt=(nx, ny), divV=(nx, ny), txx=(nx, ny), tyy=(nx, ny), txy=(nx - 1, ny - 1),
                   Rx=(nx - 1, ny - 2), Ry=(nx - 2, ny - 1), dVx=(nx - 1, ny - 2), dVy=(nx - 2, ny - 1),
                   Mus2=(nx, ny), Must=(nx, ny), Gdt=(nx, ny), dtRho=(nx, ny))
        if self.elastic:
            self.alloc(txx_o=(nx, ny), tyy_o=(nx, ny), txy_o=(nx - 1, ny - 1))
        dx, dy, lx, ly = self.dx, self.dy, self.lx, self.ly
        ix = np.arange(1, nx + 2, dtype=np.float64)
        iy = np.arange(1, ny + 2, dtype=np.float64)
        X = (ix[:nx] - 1) * dx + 0.5 * dx - 0.5 * lx
        Y = (iy[:ny] - 1) * dy + 0.5 * dy - 0.5 * ly
        Rad2 = np.asfortranarray(X[:, None] ** 2 + Y[None, :] ** 2)
        self.f["Vx"] = np.asfortranarray(np.repeat((-self.ebg * ((ix - 1) * dx - 0.5 * lx))[:, None], ny, axis=1))
        self.f["Vy"] = np.asfortranarray(np.repeat((self.ebg * ((iy - 1) * dy - 0.5 * ly))[None, :], nx, axis=0))
        Mus = self.mus0 * np.ones((nx, ny), order="F")
        Mus[Rad2 < 1.0] = self.musi
        self.init_viscosity(Mus)
        return self

    def init_viscosity(self, Mus):
        """Smoothing, local-max viscosity and iteration parameters (Stokes2D.jl:115-125)."""
        L = self.L
        Mus2 = self.f["Mus2"]
        Mus2[...] = Mus
        for _ in range(10):
            L.ora2_smooth(arr(Mus2), arr(Mus), 1.0)
            Mus, Mus2 = Mus2, Mus
        self.f["Mus"], self.f["Mus2"] = Mus, Mus2
        Must = self.f["Must"]
        Must[...] = Mus
        L.ora2_maxloc(arr(Must), arr(Mus))
        L.ora2_bc_x(arr(Must))
        L.ora2_bc_y(arr(Must))
        self.iter_params()

    def bc(self):
        self.L.ora2_bc_y(self.A("Vx"))
        self.L.ora2_bc_x(self.A("Vy"))

    def assign_tau(self):
        for n in ("txx", "tyy", "txy"):
            self.L.ora_copy(self.A(n + "_o"), self.A(n))


class V2D(_Case2D):
    """scripts/Stokes2D.jl (2D viscous)."""

    elastic = False
    defaults = dict(nt=1, iterMax=1e5, nout=500, eps=1e-8, CFL=0.9 / math.sqrt(2), Re=5 * PI, r=1.0)

    def iter_params(self):
        self.L.ora_iter_params_v(self.A("dtRho"), self.A("Gdt"), self.A("Must"), self.Vpdt, self.Re, self.r,
                                 self.max_lxy)

    def iteration(self):
        L, A = self.L, self.A
        L.ora2_compute_P(A("divV"), A("Pt"), A("Vx"), A("Vy"), A("Gdt"), self.r, self.dx, self.dy)
        L.ora2v_compute_tau(A("txx"), A("tyy"), A("txy"), A("Vx"), A("Vy"), A("Mus"), A("Gdt"), self.dx, self.dy)
        L.ora2v_compute_dV(A("Rx"), A("Ry"), A("dVx"), A("dVy"), A("Pt"), A("txx"), A("tyy"), A("txy"),
                           A("dtRho"), self.dx, self.dy)
        L.ora2_compute_V(A("Vx"), A("Vy"), A("dVx"), A("dVy"))
        self.bc()

    def check(self):
        # Rx, Ry come from compute_dV! of this iteration (Stokes2D.jl:136-143)
        return self.norm_err(("Rx", "Ry"), "divV")


class V2DSweep(V2D):
    """One instance of the batched 2D viscous sweep, with the numerics of the reference's
    sweep script scripts/Stokes2D_param.jl: its compute_τ! form
    τ = 2μ_veτ(ε̇ + τ/Gdτ/2), μ_veτ = 1/(1/Gdτ + 1/Mus) (:48-55), its buoyancy term
    Ry -= @av_yi(ρg) (:59), and uniform iteration parameters from Musτ .= μs0 (:190-192), so
    Gdτ and dτ_Rho hold one value per instance; a box lx = aspect*ly
    (scripts/Stokes2D_ve_param.jl:99-102); one centred circular inclusion of radius 1 with
    viscosity musi and density contrast rhogi; pure shear ebg; Mus and ρg smoothed alike
    (Stokes2D_param.jl:184-189); iterMax = 100max(nx,ny) unless given (:146). The check is
    Stokes2D_param.jl's (Vmin/Vmax over Vy, :204-208) with the norms scaled by ly
    (Stokes2D_ve_param.jl:175-176) and a single tolerance on max(norm_Rx, norm_Ry, norm_∇V).

    Stokes2D.jl's own form (iteration parameters from the local maxloc of Mus) diverges at
    the sweep's strongest contrasts (musi ~ 1e-5..1e-6 on 255 and 511 cells); the param
    script's uniform parameters do not."""

    defaults = dict(nt=1, iterMax=None, nout=200, eps=1e-8, CFL=0.9 / math.sqrt(2), Re=5 * PI, r=1.0, rhogi=0.0)

    def setup(self):
        nx, ny = self.nx, self.ny
        if self.iterMax is None:
            self.iterMax = 100 * max(nx, ny)
        self.ly = 10.0 if "ly" not in self.p else self.p["ly"]
        self.dx, self.dy = self.lx / nx, self.ly / ny
        self._dx, self._dy = 1.0 / self.dx, 1.0 / self.dy
        self.max_lxy = max(self.lx, self.ly)
        self.Vpdt = min(self.dx, self.dy) * self.CFL
        self.xc = linrange(self.dx / 2, self.lx - self.dx / 2, nx)
        self.yc = linrange(self.dy / 2, self.ly - self.dy / 2, ny)
        self.alloc(Pt=(nx, ny), divV=(nx, ny), txx=(nx, ny), tyy=(nx, ny), txy=(nx - 1, ny - 1),
                   Rx=(nx - 1, ny - 2), Ry=(nx - 2, ny - 1), dVx=(nx - 1, ny - 2), dVy=(nx - 2, ny - 1),
                   Mus2=(nx, ny), Must=(nx, ny), Gdt=(nx, ny), dtRho=(nx, ny), rhog2=(nx, ny))
        dx, dy, lx, ly = self.dx, self.dy, self.lx, self.ly
        ix = np.arange(1, nx + 2, dtype=np.float64)
        iy = np.arange(1, ny + 2, dtype=np.float64)
        X = (ix[:nx] - 1) * dx + 0.5 * dx - 0.5 * lx
        Y = (iy[:ny] - 1) * dy + 0.5 * dy - 0.5 * ly
        Rad2 = np.asfortranarray(X[:, None] ** 2 + Y[None, :] ** 2)
        self.f["Vx"] = np.asfortranarray(np.repeat((-self.ebg * ((ix - 1) * dx - 0.5 * lx))[:, None], ny, axis=1))
        self.f["Vy"] = np.asfortranarray(np.repeat((self.ebg * ((iy - 1) * dy - 0.5 * ly))[None, :], nx, axis=0))
        Mus = self.mus0 * np.ones((nx, ny), order="F")
        Mus[Rad2 < 1.0] = self.musi
        rhog = np.zeros((nx, ny), order="F")
        rhog[Rad2 < 1.0] = self.rhogi
        L = self.L
        Mus2, rhog2 = self.f["Mus2"], self.f["rhog2"]
        Mus2[...] = Mus
        rhog2[...] = rhog
        for _ in range(10):
            L.ora2_smooth(arr(Mus2), arr(Mus), 1.0)
            Mus, Mus2 = Mus2, Mus
            L.ora2_smooth(arr(rhog2), arr(rhog), 1.0)
            rhog, rhog2 = rhog2, rhog
        self.f["Mus"], self.f["Mus2"], self.f["rhog"], self.f["rhog2"] = Mus, Mus2, rhog, rhog2
        self.f["Must"][...] = self.mus0  # Musτ .= μs0
        self.iter_params()
        return self

    def iteration(self):
        L, A = self.L, self.A
        L.ora2_compute_P(A("divV"), A("Pt"), A("Vx"), A("Vy"), A("Gdt"), self.r, self.dx, self.dy)
        L.ora2s_compute_tau(A("txx"), A("tyy"), A("txy"), A("Vx"), A("Vy"), A("Mus"), A("Gdt"), self.dx, self.dy)
        L.ora2s_compute_dV(A("Rx"), A("Ry"), A("dVx"), A("dVy"), A("Pt"), A("txx"), A("tyy"), A("txy"),
                           A("dtRho"), A("rhog"), self.dx, self.dy)
        L.ora2_compute_V(A("Vx"), A("Vy"), A("dVx"), A("dVy"))
        self.bc()

    def check(self):
        _, vmin, vmax = stats(self.f["Vy"])
        _, pmin, pmax = stats(self.f["Pt"])
        norms = []
        for n in ("Rx", "Ry"):
            s, _, _ = stats(self.f[n])
            norms.append(math.sqrt(s) / (pmax - pmin) * self.ly / math.sqrt(self.f[n].size))
        s, _, _ = stats(self.f["divV"])
        norms.append(math.sqrt(s) / (vmax - vmin) * self.ly / math.sqrt(self.f["divV"].size))
        return max(norms), norms


class VE2D(_Case2D):
    """scripts/Stokes2D_ve.jl (2D Maxwell visco-elastic, role kernels)."""

    defaults = dict(nt=5, iterMax=2e5, nout=200, eps=1e-8, CFL=0.8 / math.sqrt(2), Re=5 * PI, r=1.0)

    def iter_params(self):
        self.L.ora_iter_params_ve(self.A("dtRho"), self.A("Gdt"), self.A("Must"), self.Vpdt, self.G, self.dt,
                                  self.Re, self.r, self.max_lxy)

    def iteration(self):
        L, A = self.L, self.A
        L.ora2_compute_P(A("divV"), A("Pt"), A("Vx"), A("Vy"), A("Gdt"), self.r, self.dx, self.dy)
        L.ora2ve_compute_tau(A("txx"), A("tyy"), A("txy"), A("txx_o"), A("tyy_o"), A("txy_o"), A("Gdt"), A("Vx"),
                             A("Vy"), A("Mus"), self.G, self.dt, self.dx, self.dy)
        L.ora2ve_compute_dV(A("dVx"), A("dVy"), A("Pt"), A("txx"), A("tyy"), A("txy"), A("dtRho"), self.dx, self.dy)
        L.ora2_compute_V(A("Vx"), A("Vy"), A("dVx"), A("dVy"))
        self.bc()

    def check(self):
        A = self.A
        self.L.ora2ve_compute_Res(A("Rx"), A("Ry"), A("Pt"), A("txx"), A("tyy"), A("txy"), self.dx, self.dy)
        return self.norm_err(("Rx", "Ry"), "divV")


class VE2DParam(VE2D):
    """scripts/Stokes2D_ve_param.jl, the aspect-ratio study (2D Maxwell VE, role kernels):
    ly = 10, lx = nsub*ly, nx = nsub*(ny+1)-1 (:99-107), nsub inclusions of radius 1 along x
    (:138-141), min_lxy = fact*min(lx,ly) in the iteration parameters (:110, :150), CFL
    0.87/sqrt(2), eps = 1e-6, iterMax = 100nx, nout = nx (:103-109), and norm_Rx scaled by lx,
    norm_Ry and norm_∇V by ly (:175-177)."""

    defaults = dict(nt=5, eps=1e-6, CFL=0.87 / math.sqrt(2), Re=5 * PI, r=1.0, nsub=1, fact=1.0, ly=10.0)

    def __init__(self, ny, nsub=1, fact=1.0, **kw):
        ly = kw.pop("ly", 10.0)
        nx = nsub * (ny + 1) - 1
        super().__init__(nx, ny, None, ly=ly, lx=nsub * ly, nsub=nsub, fact=fact, **kw)
        self.iterMax = 100 * nx
        self.nout = nx

    def setup(self):
        super().setup()  # allocations, the script's Vx/Vy; Mus replaced below
        nx, ny, dx, dy, ly = self.nx, self.ny, self.dx, self.dy, self.ly
        ix = np.arange(1, nx + 1, dtype=np.float64)
        iy = np.arange(1, ny + 1, dtype=np.float64)
        Mus = self.mus0 * np.ones((nx, ny), order="F")
        for isub in range(1, self.nsub + 1):
            X = (ix - 1) * dx + 0.5 * dx - 0.5 * ly - (isub - 1) * ly
            Y = (iy - 1) * dy + 0.5 * dy - 0.5 * ly
            Rad2 = X[:, None] ** 2 + Y[None, :] ** 2
            Mus[Rad2 < 1.0] = self.musi
        for k in ("Pt", "divV", "txx", "tyy", "txy", "txx_o", "tyy_o", "txy_o"):
            self.f[k][...] = 0.0
        self.init_viscosity(Mus)
        return self

    def iter_params(self):
        min_lxy = self.fact * min(self.lx, self.ly)
        self.L.ora_iter_params_ve(self.A("dtRho"), self.A("Gdt"), self.A("Must"), self.Vpdt, self.G, self.dt,
                                  self.Re, self.r, min_lxy)

    def check(self):
        A = self.A
        self.L.ora2ve_compute_Res(A("Rx"), A("Ry"), A("Pt"), A("txx"), A("tyy"), A("txy"), self.dx, self.dy)
        _, vmin, vmax = stats(self.f["Vx"])
        _, pmin, pmax = stats(self.f["Pt"])
        norms = []
        for n, L in (("Rx", self.lx), ("Ry", self.ly)):
            sq, _, _ = stats(self.f[n])
            norms.append(math.sqrt(sq) / (pmax - pmin) * L / math.sqrt(self.f[n].size))
        sq, _, _ = stats(self.f["divV"])
        norms.append(math.sqrt(sq) / (vmax - vmin) * self.ly / math.sqrt(self.f["divV"].size))
        return max(norms), norms

    def output_line(self):
        """The script's result line (`println(io, "$(nx) $(ny) $(nsub) $(fact) $(ittot) $(nt) $(err)")`)."""
        return self.nx, self.ny, self.nsub, self.fact, self.ittot, self.nt


class VE2DPerf(VE2D):
    """scripts/Stokes2D_ve_perf.jl (2D VE, fused explicit-index kernels)."""

    defaults = dict(nt=1, iterMax=100, nout=2000, eps=1e-8, CFL=0.8 / math.sqrt(2), Re=5 * PI, r=1.0)

    def iteration(self):
        L, A = self.L, self.A
        L.ora2p_compute_Pt_tau(A("Pt"), A("txx"), A("tyy"), A("txy"), A("txx_o"), A("tyy_o"), A("txy_o"), A("Gdt"),
                               A("Vx"), A("Vy"), A("Mus"), self.r, self.G, self.dt, self._dx, self._dy)
        Vx, Vy = self.f["Vx"], self.f["Vy"]
        L.ora2p_compute_V(A("Vx"), A("Vy"), A("Pt"), A("txx"), A("tyy"), A("txy"), A("dtRho"), self._dx, self._dy,
                          Vx.shape[0] - 2, Vx.shape[1] - 2, Vy.shape[0] - 2, Vy.shape[1] - 2)
        self.bc()

    def check(self):
        A = self.A
        self.L.ora2p_compute_Res(A("divV"), A("Rx"), A("Ry"), A("Pt"), A("Vx"), A("Vy"), A("txx"), A("tyy"),
                                 A("txy"), self._dx, self._dy)
        return self.norm_err(("Rx", "Ry"), "divV")


class VE2DDamp(_Case2D):
    """scripts/previous_damp/Stokes2D_ve0.jl (2D Maxwell VE, the damped "accel. 1" scheme):
    numerical compressibility β_n in τ, a damped rate dV/dτ = damp*dV/dτ + R and per-face
    pseudo-time steps dτV = min(dx,dy)^2/4.1/Vsc/@av(Musτ)/(1+β_n), dτPt = 4.1(1+β_n)/Ptsc/
    max(nx,ny)*Musτ (:27-32). Set-up and initial conditions are Stokes2D.jl's (:118-145); the
    check is the same (Vmin/Vmax over Vx, norms scaled by lx, :160-167)."""

    defaults = dict(nt=5, iterMax=2e5, nout=200, eps=1e-8, Vdmp=4.0, beta_n=2.0, Vsc=1.0, Ptsc=3.0, CFL=0.0,
                    Re=0.0, r=0.0, err_form="scaled")

    def setup(self):
        nx, ny = self.nx, self.ny
        self.dampX, self.dampY = 1.0 - self.Vdmp / nx, 1.0 - self.Vdmp / ny
        # dVx/dVy hold the damped rates dVxdτ/dVydτ: zero at start, carried across time steps
        return super().setup()

    def iter_params(self):
        nx, ny = self.nx, self.ny
        self.alloc(dtVx=(nx - 1, ny - 2), dtVy=(nx - 2, ny - 1), dtPt=(nx, ny))
        self.L.ora2d_timesteps(self.A("dtVx"), self.A("dtVy"), self.A("dtPt"), self.A("Must"), self.Vsc, self.Ptsc,
                               min(self.dx, self.dy) ** 2, self.beta_n, float(max(nx, ny)))

    def iteration(self):
        L, A = self.L, self.A
        L.ora2d_compute_P(A("divV"), A("Pt"), A("Vx"), A("Vy"), A("dtPt"), self.dx, self.dy)
        o = (A("txx_o"), A("tyy_o"), A("txy_o")) if self.elastic else (A("txx"), A("tyy"), A("txy"))
        L.ora2d_compute_tau(A("txx"), A("tyy"), A("txy"), *o, A("Vx"), A("Vy"), A("Mus"), A("divV"), self.G, self.dt,
                            self.beta_n, self.dx, self.dy, int(self.elastic))
        L.ora2d_compute_dV(A("Rx"), A("Ry"), A("dVx"), A("dVy"), A("Pt"), A("txx"), A("tyy"), A("txy"), self.dampX,
                           self.dampY, self.dx, self.dy)
        L.ora2d_compute_V(A("Vx"), A("Vy"), A("dVx"), A("dVy"), A("dtVx"), A("dtVy"))
        self.bc()

    def check(self):
        """err of the check (Stokes2D_ve0.jl:160-167; Rx, Ry come from compute_dV! of this
        iteration). err_form "scaled" is the script's active measure (:163-165): ||R||_2
        scaled by the pressure or velocity range, lx and 1/sqrt(length). err_form "length" is
        the measure the script keeps commented out beside it (:166), ||R||_2 / length(R) for
        Rx, Ry and ∇V: with it the restatement takes exactly the iteration totals of the
        reference's output/out_Stokes2D_ve0.txt (2800, 4800, 9000, 16800 at 31^2 .. 255^2)."""
        if self.err_form == "scaled":
            return self.norm_err(("Rx", "Ry"), "divV")
        if self.err_form != "length":
            raise ValueError(f"err_form must be 'scaled' or 'length', not {self.err_form!r}")
        norms = []
        for n in ("Rx", "Ry", "divV"):
            s, _, _ = stats(self.f[n])
            norms.append(math.sqrt(s) / self.f[n].size)
        return max(norms), norms


class V2DDamp(VE2DDamp):
    """scripts/previous_damp/Stokes2D0.jl (2D viscous, damped scheme): VE2DDamp without
    the elastic terms, τ = 2Mus(ε̇ - ∇V/3 + β_n ∇V) (:39-44); one solve, iterMax 1e5,
    nout 500 (:79-80)."""

    elastic = False
    defaults = dict(VE2DDamp.defaults, nt=1, iterMax=1e5, nout=500)


class _Case3D(Case):
    ndim = 3
    igg_coords = False  # Stokes3D_ve_multixpu.jl builds the ICs through ImplicitGlobalGrid's x_g

    def setup(self):
        """Allocations, initial conditions and iteration parameters (Stokes3D_ve_perf.jl:135-192)."""
        nx, ny, nz = self.nx, self.ny, self.nz
        self.dx, self.dy, self.dz = self.lx / nx, self.ly / ny, self.lz / nz
        self._dx, self._dy, self._dz = 1.0 / self.dx, 1.0 / self.dy, 1.0 / self.dz
        self.max_lxyz = max(self.lx, self.ly, self.lz)
        self.Vpdt = min(self.dx, self.dy, self.dz) * self.CFL
        self.xc = linrange(self.dx / 2, self.lx - self.dx / 2, nx)
        self.yc = linrange(self.dy / 2, self.ly - self.dy / 2, ny)
        self.zc = linrange(self.dz / 2, self.lz - self.dz / 2, nz)
        self.alloc(Pt=(nx, ny, nz), dtRho=(nx, ny, nz), Gdt=(nx, ny, nz), divV=(nx, ny, nz), Vy=(nx, ny + 1, nz),
                   txx=(nx, ny - 2, nz - 2), tyy=(nx - 2, ny, nz - 2), tzz=(nx - 2, ny - 2, nz),
                   txy=(nx - 1, ny - 1, nz - 2), txz=(nx - 1, ny - 2, nz - 1), tyz=(nx - 2, ny - 1, nz - 1),
                   Rx=(nx - 1, ny - 2, nz - 2), Ry=(nx - 2, ny - 1, nz - 2), Rz=(nx - 2, ny - 2, nz - 1),
                   Mus2=(nx, ny, nz), Must=(nx, ny, nz))
        if self.elastic:
            for n in ("txx", "tyy", "tzz", "txy", "txz", "tyz"):
                self.f[n + "_o"] = zeros(*self.f[n].shape)
        if self.unfused:
            self.alloc(dVx=(nx - 1, ny - 2, nz - 2), dVy=(nx - 2, ny - 1, nz - 2), dVz=(nx - 2, ny - 2, nz - 1))
        dx, dy, dz, lx, ly, lz = self.dx, self.dy, self.dz, self.lx, self.ly, self.lz
        ix = np.arange(1, nx + 2, dtype=np.float64)
        iy = np.arange(1, ny + 1, dtype=np.float64)
        iz = np.arange(1, nz + 2, dtype=np.float64)
        X = (ix[:nx] - 1) * dx + 0.5 * dx - 0.5 * lx
        Y = (iy - 1) * dy + 0.5 * dy - 0.5 * ly
        Z = (iz[:nz] - 1) * dz + 0.5 * dz - 0.5 * lz
        if self.igg_coords:
            # x_g(ix,dx,A) = (ix-1)*dx + 0.5*(nx_g-size(A,1))*dx (ImplicitGlobalGrid, 1 rank);
            # for the staggered Vx/Vz this is (ix-1)*dx - 0.5*dx (Stokes3D_ve_multixpu.jl:174-176).
            xv = ((ix - 1) * dx + (-0.5 * dx)) + 0.5 * dx - 0.5 * lx
            zv = ((iz - 1) * dz + (-0.5 * dz)) + 0.5 * dz - 0.5 * lz
            X = ((ix[:nx] - 1) * dx + 0.0) + 0.5 * dx - 0.5 * lx
            Y = ((iy - 1) * dy + 0.0) + 0.5 * dy - 0.5 * ly
            Z = ((iz[:nz] - 1) * dz + 0.0) + 0.5 * dz - 0.5 * lz
        else:
            xv = (ix - 1) * dx - 0.5 * lx
            zv = (iz - 1) * dz - 0.5 * lz
        Rad2 = (X[:, None, None] ** 2 + Y[None, :, None] ** 2) + Z[None, None, :] ** 2
        self.f["Vx"] = np.asfortranarray(np.broadcast_to((-self.ebg * xv)[:, None, None], (nx + 1, ny, nz)))
        self.f["Vz"] = np.asfortranarray(np.broadcast_to((self.ebg * zv)[None, None, :], (nx, ny, nz + 1)))
        Mus = self.mus0 * np.ones((nx, ny, nz), order="F")
        Mus[Rad2 < 1.0] = self.musi
        self.init_viscosity(Mus)
        return self

    def init_viscosity(self, Mus):
        """Smoothing, local-max viscosity and iteration parameters (Stokes3D_ve_perf.jl:173-192)."""
        L = self.L
        Mus = np.asfortranarray(Mus, dtype=np.float64)
        Mus2 = self.f["Mus2"]
        Mus2[...] = Mus
        for _ in range(10):
            L.ora3_smooth(arr(Mus2), arr(Mus), 1.0)
            Mus, Mus2 = Mus2, Mus
        self.f["Mus"], self.f["Mus2"] = Mus, Mus2
        Must = self.f["Must"]
        Must[...] = Mus
        L.ora3_maxloc(arr(Must), arr(Mus))
        L.ora3_bc_x(arr(Must))
        L.ora3_bc_y(arr(Must))
        L.ora3_bc_z(arr(Must))
        self.iter_params()

    def iter_params(self):
        if self.elastic:
            self.L.ora_iter_params_ve(self.A("dtRho"), self.A("Gdt"), self.A("Must"), self.Vpdt, self.G, self.dt,
                                      self.Re, self.r, self.max_lxyz)
        else:
            self.L.ora_iter_params_v(self.A("dtRho"), self.A("Gdt"), self.A("Must"), self.Vpdt, self.Re, self.r,
                                     self.max_lxyz)

    def bc(self):
        """The six free-slip copies, in the reference's order (Stokes3D_ve_perf.jl:202-207)."""
        L, A = self.L, self.A
        L.ora3_bc_x(A("Vy"))
        L.ora3_bc_x(A("Vz"))
        L.ora3_bc_y(A("Vx"))
        L.ora3_bc_y(A("Vz"))
        L.ora3_bc_z(A("Vx"))
        L.ora3_bc_z(A("Vy"))

    def assign_tau(self):
        for n in ("txx", "tyy", "tzz", "txy", "txz", "tyz"):
            self.L.ora_copy(self.A(n + "_o"), self.A(n))

    def _tau_o(self):
        if self.elastic:
            return [self.A(n + "_o") for n in ("txx", "tyy", "tzz", "txy", "txz", "tyz")]
        return [arr(None)] * 6

    def _tau(self):
        return [self.A(n) for n in ("txx", "tyy", "tzz", "txy", "txz", "tyz")]


class VE3D(_Case3D):
    """scripts/stokes_3D/Stokes3D_ve_multixpu.jl on one rank (role kernels, /dx form)."""

    unfused = True
    igg_coords = True
    defaults = dict(nt=5, iterMax=2e5, nout=200, eps=1e-8, CFL=0.8 / math.sqrt(3), Re=6 * PI, r=1.0)

    def iteration(self):
        L, A = self.L, self.A
        L.ora3m_compute_P(A("divV"), A("Pt"), A("Vx"), A("Vy"), A("Vz"), A("Gdt"), self.r, self.dx, self.dy, self.dz)
        L.ora3m_compute_tau(*self._tau(), *self._tau_o(), A("Vx"), A("Vy"), A("Vz"), A("Mus"), A("Gdt"), self.G,
                            self.dt, self.dx, self.dy, self.dz, int(self.elastic))
        L.ora3m_compute_dV(A("dVx"), A("dVy"), A("dVz"), A("Pt"), *self._tau(), A("dtRho"), self.dx, self.dy,
                           self.dz, 0)
        L.ora3_compute_V(A("Vx"), A("Vy"), A("Vz"), A("dVx"), A("dVy"), A("dVz"))
        self.bc()

    def check(self):
        A = self.A
        self.L.ora3m_compute_dV(A("Rx"), A("Ry"), A("Rz"), A("Pt"), *self._tau(), arr(None), self.dx, self.dy,
                                self.dz, 1)
        return self.norm_err(("Rx", "Ry", "Rz"), "divV")


class V3DDamp(_Case3D):
    """scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl on one rank (3D viscous, the damped
    "accel. 1" scheme): β_n in τ, a damped rate dV/dτ = damp*dV/dτ + R, per-face pseudo-time
    steps (:37-43); ICs through ImplicitGlobalGrid's x_g as Stokes3D_ve_multixpu.jl
    (:144-166); one solve, iterMax 6e4, nout 500, Vdmp 4, β_n 3, Vsc 1, Ptsc 5 (:102-109);
    the check of Stokes3D_ve_multixpu.jl on one rank (:206-216)."""

    elastic = False
    unfused = True
    igg_coords = True
    defaults = dict(nt=1, iterMax=6e4, nout=500, eps=1e-8, Vdmp=4.0, beta_n=3.0, Vsc=1.0, Ptsc=5.0, CFL=0.0,
                    Re=0.0, r=0.0)

    def iter_params(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        self.dampX, self.dampY, self.dampZ = 1.0 - self.Vdmp / nx, 1.0 - self.Vdmp / ny, 1.0 - self.Vdmp / nz
        self.alloc(dtVx=self.f["Rx"].shape, dtVy=self.f["Ry"].shape, dtVz=self.f["Rz"].shape, dtPt=(nx, ny, nz))
        self.L.ora3d_timesteps(self.A("dtVx"), self.A("dtVy"), self.A("dtVz"), self.A("dtPt"), self.A("Must"),
                               self.Vsc, self.Ptsc, min(self.dx, self.dy, self.dz) ** 2, self.beta_n,
                               float(max(nx, ny, nz)))

    def iteration(self):
        L, A = self.L, self.A
        L.ora3d_compute_P(A("divV"), A("Pt"), A("Vx"), A("Vy"), A("Vz"), A("dtPt"), self.dx, self.dy, self.dz)
        L.ora3d_compute_tau(A("divV"), *self._tau(), A("Vx"), A("Vy"), A("Vz"), A("Mus"), self.beta_n, self.dx,
                            self.dy, self.dz)
        L.ora3d_compute_dV(A("Rx"), A("Ry"), A("Rz"), A("dVx"), A("dVy"), A("dVz"), A("Pt"), *self._tau(),
                           self.dampX, self.dampY, self.dampZ, self.dx, self.dy, self.dz)
        L.ora3d_compute_V(A("Vx"), A("Vy"), A("Vz"), A("dVx"), A("dVy"), A("dVz"), A("dtVx"), A("dtVy"), A("dtVz"))
        self.bc()

    def check(self):
        # Rx, Ry, Rz from compute_dV! of this iteration (Stokes3D0_multixpu.jl:206-213)
        return self.norm_err(("Rx", "Ry", "Rz"), "divV")


class VE3DPerf(_Case3D):
    """scripts/stokes_3D/Stokes3D_ve_perf.jl (fused explicit-index kernels, _dx form).

    Adjoint support (no reference counterpart): momentum sources F added to the residual
    (set_sources); with adjoint=True the case iterates the transposed system: the free-slip
    ghosts stay zero and each ghost face's residual is added to the interior face it copies
    (ora3v_res_adj). grad_logmu_ve gives one visco-elastic step's ∂J/∂log μ term from this
    (forward) case's stresses and an adjoint case's stresses."""

    unfused = False
    defaults = dict(nt=1, iterMax=200, nout=2000, eps=1e-8, CFL=0.8 / math.sqrt(3), Re=6 * PI, r=1.0,
                    adjoint=False)

    def clear_state(self):
        """Zero V, Pt and τ (walls and ghosts included): the adjoint's initial state."""
        for n in ("Pt", "Vx", "Vy", "Vz", "txx", "tyy", "tzz", "txy", "txz", "tyz"):
            self.f[n][...] = 0.0

    def set_sources(self, Fx, Fy, Fz):
        for name, a in (("Fx", Fx), ("Fy", Fy), ("Fz", Fz)):
            assert a.shape == self.f["R" + name[1]].shape
            self.f[name] = np.asfortranarray(a, dtype=np.float64)

    def iteration(self):
        L, A = self.L, self.A
        L.ora3p_compute_Pt_tau(A("Pt"), *self._tau(), *self._tau_o(), A("Vx"), A("Vy"), A("Vz"), A("Mus"), A("Gdt"),
                               self.r, self.G, self.dt, self._dx, self._dy, self._dz, int(self.elastic))
        if self.adjoint:
            if "Fx" not in self.f:
                self.set_sources(*(np.zeros_like(self.f["R" + c]) for c in "xyz"))
            L.ora3v_res_adj(A("Rx"), A("Ry"), A("Rz"), A("Pt"), *self._tau(), self._dx, self._dy, self._dz)
            L.ora3v_update_V(A("Vx"), A("Vy"), A("Vz"), A("Rx"), A("Ry"), A("Rz"), A("Fx"), A("Fy"), A("Fz"),
                             A("dtRho"))
            return
        if "Fx" in self.f:
            L.ora3p_compute_V_src(A("Vx"), A("Vy"), A("Vz"), A("Pt"), *self._tau(), A("dtRho"), A("Fx"), A("Fy"),
                                  A("Fz"), self._dx, self._dy, self._dz)
        else:
            L.ora3p_compute_V(A("Vx"), A("Vy"), A("Vz"), A("Pt"), *self._tau(), A("dtRho"), self._dx, self._dy,
                              self._dz)
        self.bc()

    def check(self):
        A = self.A
        self.L.ora3p_compute_Res(A("divV"), A("Rx"), A("Ry"), A("Rz"), A("Vx"), A("Vy"), A("Vz"), A("Pt"),
                                 *self._tau(), self._dx, self._dy, self._dz)
        if self.adjoint:
            self.L.ora3v_res_adj(A("Rx"), A("Ry"), A("Rz"), A("Pt"), *self._tau(), self._dx, self._dy, self._dz)
        if "Fx" in self.f:
            for c in "xyz":
                self.f["R" + c][...] = self.f["R" + c] + self.f["F" + c]
        return self.norm_err(("Rx", "Ry", "Rz"), "divV")

    def grad_logmu_ve(self, adj, out=None, tau=None):
        """One visco-elastic step's ∂J/∂log μ term: written into a new array, or added to
        `out`. `tau` (6 arrays) replaces this case's current stresses (a checkpoint)."""
        add = out is not None
        g = out if add else zeros(self.nx, self.ny, self.nz)
        T = [arr(t) for t in tau] if tau is not None else self._tau()
        self.L.ora3ve_grad_logmu(arr(g), *T, *adj._tau(), self.A("Mus"), int(add))
        return g


class V3D(VE3DPerf):
    """3D viscous Stokes: the fused 3D kernels without elastic terms (no reference script).

    Adjoint support as in VE3DPerf, plus one application of the operator -- τ = 2με̇(V),
    then R = ∇·τ − ∇P + F and ∇V (apply_operator) -- and the viscous ∂J/∂log μ from this
    case's V and an adjoint case's V (grad_logmu)."""

    elastic = False
    defaults = dict(nt=1, iterMax=2e5, nout=200, eps=1e-8, CFL=0.8 / math.sqrt(3), Re=6 * PI, r=1.0,
                    adjoint=False)

    def apply_operator(self):
        A = self.A
        self.L.ora3v_tau_exact(*self._tau(), A("Vx"), A("Vy"), A("Vz"), A("Mus"), self._dx, self._dy, self._dz)
        return self.check()

    def grad_logmu(self, adj):
        g = zeros(self.nx, self.ny, self.nz)
        A, B = self.A, adj.A
        self.L.ora3v_grad_logmu(arr(g), A("Vx"), A("Vy"), A("Vz"), B("Vx"), B("Vy"), B("Vz"), A("Mus"), self._dx,
                                self._dy, self._dz)
        return g


VARIANTS = {
    "2d_v": V2D,
    "2d_ve": VE2D,
    "2d_ve_perf": VE2DPerf,
    "3d_ve": VE3D,
    "3d_ve_perf": VE3DPerf,
    "3d_v": V3D,
    "2d_v_damp": V2DDamp,
    "2d_ve_damp": VE2DDamp,
    "3d_v_damp": V3DDamp,
}


def make(variant, nx, ny, nz=None, **kw):
    return VARIANTS[variant](nx, ny, nz, **kw).setup()


def fixture_sample(case):
    """The reference test's sample: 12 indices per dimension (test/test_2D.jl:19-21)."""
    def inds(n):
        return (np.ceil(linrange(1.0, float(n), 12)).astype(np.int64) - 1)
    ix = inds(case.nx)
    iy = inds(case.ny)
    if case.ndim == 2:
        P = case.f["Pt"][np.ix_(ix, iy)]
    else:
        iz = inds(case.nz)
        P = case.f["Pt"][np.ix_(ix, iy, iz)]
    return case.xc[ix], P
