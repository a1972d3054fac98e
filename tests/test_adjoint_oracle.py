"""The adjoint of the 3D viscous solve, checked on the oracle alone (no GPU).

The oracle's transposed system (zero ghosts, ghost residuals folded onto the faces they
copy) must satisfy <A(u,p), (w,q)> = <(u,p), Aᵀ(w,q)> to rounding, and the adjoint
∂J/∂log μ must match central finite differences of J = ½‖Vz(top) − Vobs‖²."""
import math

import numpy as np

from oracle import scripts as S

NX, NY, NZ = 11, 10, 9


def case(adjoint=False, mus=None, eps=1e-12):
    o = S.V3D(NX, NY, NZ, musi=1e-2, nout=100, eps=eps, iterMax=3e5, adjoint=adjoint).setup()
    if mus is not None:
        o.f["Mus"][...] = mus
    if adjoint:
        o.clear_state()
    return o


def random_state(o, rng, copies):
    o.clear_state()
    o.f["Vx"][1:NX, 1:NY - 1, 1:NZ - 1] = rng.standard_normal((NX - 1, NY - 2, NZ - 2))
    o.f["Vy"][1:NX - 1, 1:NY, 1:NZ - 1] = rng.standard_normal((NX - 2, NY - 1, NZ - 2))
    o.f["Vz"][1:NX - 1, 1:NY - 1, 1:NZ] = rng.standard_normal((NX - 2, NY - 2, NZ - 1))
    if copies:
        o.bc()
    o.f["Pt"][...] = rng.standard_normal((NX, NY, NZ))
    return (o.f["Vx"][1:NX, 1:NY - 1, 1:NZ - 1].copy(), o.f["Vy"][1:NX - 1, 1:NY, 1:NZ - 1].copy(),
            o.f["Vz"][1:NX - 1, 1:NY - 1, 1:NZ].copy(), o.f["Pt"].copy())


def top(o):
    return o.f["Vz"][1:NX - 1, 1:NY - 1, NZ - 1].copy()


def test_transposed_system_satisfies_the_dot_product_identity():
    rng = np.random.default_rng(3)
    fw, ad = case(), case(adjoint=True)
    u = random_state(fw, rng, copies=True)
    fw.apply_operator()
    Au = [fw.f[n].copy() for n in ("Rx", "Ry", "Rz", "divV")]
    w = random_state(ad, rng, copies=False)
    ad.apply_operator()
    Atw = [ad.f[n].copy() for n in ("Rx", "Ry", "Rz", "divV")]
    lhs = sum(float(np.sum(a * b)) for a, b in zip(Au, w))
    rhs = sum(float(np.sum(a * b)) for a, b in zip(u, Atw))
    assert abs(lhs - rhs) <= 1e-13 * abs(lhs)
    # without the fold the operator is not symmetric: the identity fails
    plain = case()
    plain.f["Vx"][...] = ad.f["Vx"]
    plain.f["Vy"][...] = ad.f["Vy"]
    plain.f["Vz"][...] = ad.f["Vz"]
    plain.f["Pt"][...] = ad.f["Pt"]
    plain.apply_operator()
    Kw = [plain.f[n].copy() for n in ("Rx", "Ry", "Rz", "divV")]
    rhs_plain = sum(float(np.sum(a * b)) for a, b in zip(u, Kw))
    assert abs(lhs - rhs_plain) > 1e-6 * abs(lhs)


def test_adjoint_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    f0 = case()
    mus0 = f0.f["Mus"].copy()
    f0.run()
    vobs = top(f0) + 0.1 * rng.standard_normal(top(f0).shape)

    def J(o):
        r = top(o) - vobs
        return 0.5 * float(np.sum(r * r))

    a = case(adjoint=True)
    Fz = np.zeros((NX - 2, NY - 2, NZ - 1), order="F")
    Fz[:, :, NZ - 2] = top(f0) - vobs
    a.set_sources(np.zeros((NX - 1, NY - 2, NZ - 2)), np.zeros((NX - 2, NY - 1, NZ - 2)), Fz)
    a.run()
    g = f0.grad_logmu(a)
    h = 1e-3
    for c in [(5, 5, 7), (3, 4, 6), (2, 2, 2), (8, 8, 7)]:
        Js = []
        for sgn in (1, -1):
            m = mus0.copy()
            m[c] *= math.exp(sgn * h)
            o = case(mus=m)
            o.run()
            Js.append(J(o))
        fd = (Js[0] - Js[1]) / (2 * h)
        assert abs(g[c] - fd) <= 1e-5 * abs(fd), (c, g[c], fd)


def test_visco_elastic_adjoint_over_time_steps_matches_central_differences():
    """Three Maxwell visco-elastic steps: the backward adjoint time loop (assign_τ! between
    steps, source only in the first adjoint step) with per-step stress checkpoints gives
    ∂J/∂log μ of the last step's misfit."""
    nt = 3
    tau = ("txx", "tyy", "tzz", "txy", "txz", "tyz")

    def ve(adjoint=False, mus=None):
        o = S.VE3DPerf(NX, NY, NZ, musi=1e-2, nout=100, eps=1e-12, iterMax=3e5, adjoint=adjoint).setup()
        if mus is not None:
            o.f["Mus"][...] = mus
        if adjoint:
            o.clear_state()
        return o

    def forward(o):
        cps = []
        for _ in range(nt):
            o.run(nt=1)
            cps.append([o.f[n].copy(order="F") for n in tau])
        return cps

    rng = np.random.default_rng(1)
    f0 = ve()
    mus0 = f0.f["Mus"].copy()
    cps = forward(f0)
    vobs = top(f0) + 0.1 * rng.standard_normal(top(f0).shape)
    a = ve(adjoint=True)
    Fz = np.zeros((NX - 2, NY - 2, NZ - 1), order="F")
    Fz[:, :, NZ - 2] = top(f0) - vobs
    a.set_sources(np.zeros((NX - 1, NY - 2, NZ - 2)), np.zeros((NX - 2, NY - 1, NZ - 2)), Fz)
    g = None
    for s in range(nt):
        a.run(nt=1)
        g = f0.grad_logmu_ve(a, out=g, tau=cps[nt - 1 - s])
        if s == 0:
            for c in "xyz":
                a.f["F" + c][...] = 0.0
    h = 1e-3
    for c in [(5, 5, 7), (3, 4, 6), (2, 2, 2)]:
        Js = []
        for sgn in (1, -1):
            m = mus0.copy()
            m[c] *= math.exp(sgn * h)
            o = ve(mus=m)
            forward(o)
            Js.append(0.5 * float(np.sum((top(o) - vobs) ** 2)))
        fd = (Js[0] - Js[1]) / (2 * h)
        assert abs(g[c] - fd) <= 1e-5 * abs(fd), (c, g[c], fd)
