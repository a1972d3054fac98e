"""Adjoint of the 3D viscous solve on the GPU.

The new kernels (momentum sources, the transposed system, the exact operator, the
∂J/∂log μ kernel) must equal the oracle bit for bit; the transposed system must satisfy
the dot-product identity; the gradient must match central finite differences of
J = ½‖Vz(top) − Vobs‖² at 32 random cells to 1e-5 relative; and the torch.autograd
wrapper must return the same gradient."""
import math

import numpy as np
import pytest

from oracle import scripts as S

ITER_FIELDS = ("Pt", "Vx", "Vy", "Vz", "txx", "tyy", "tzz", "txy", "txz", "tyz")


ORACLE = {"3d_v": S.V3D, "3d_ve_perf": S.VE3DPerf}


def oracle_case(n, adjoint=False, variant="3d_v", **kw):
    o = ORACLE[variant](*n, musi=1e-2, adjoint=adjoint, **kw).setup()
    if adjoint:
        o.clear_state()
    return o


def gpu_like(o, lib, adjoint=False, variant="3d_v"):
    from ptstokes import Solver
    s = Solver(variant, o.nx, o.ny, o.nz, lib=lib, adjoint=int(adjoint), nout=o.nout, eps=o.eps,
               iter_max=o.iterMax)
    s.init_inclusion(1.0, 1.0, 0.0, 0.0)
    names = ("Mus", "Must", "Gdt", "dtRho") + ITER_FIELDS
    if variant == "3d_ve_perf":
        names += tuple(n + "_o" for n in ITER_FIELDS[4:])
    for name in names:
        s.set(name, o.f[name])
    return s


def random_sources(o, rng):
    return [rng.standard_normal(o.f["R" + c].shape) for c in "xyz"]


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["3d_v", "3d_ve_perf"])
@pytest.mark.parametrize("n", [(9, 8, 7), (16, 13, 11)])
@pytest.mark.parametrize("adjoint", [False, True])
def test_iterations_with_sources_equal_the_oracle(gpu_lib, n, adjoint, variant):
    rng = np.random.default_rng(11)
    o = oracle_case(n, adjoint=adjoint, variant=variant)
    F = random_sources(o, rng)
    o.set_sources(*F)
    if variant == "3d_ve_perf":  # a pre-stress, as after assign_τ!
        for name in ITER_FIELDS[4:]:
            o.f[name + "_o"][...] = rng.standard_normal(o.f[name + "_o"].shape)
    s = gpu_like(o, gpu_lib, adjoint, variant)
    for c, a in zip("xyz", F):
        s.set("F" + c, a)
    for _ in range(37):
        o.iteration()
    s.iterate(37)
    for name in ITER_FIELDS:
        assert np.array_equal(s.get(name), o.f[name]), name
    o.check()
    s.compute_res()
    for name in ("Rx", "Ry", "Rz", "divV"):
        assert np.array_equal(s.get(name), o.f[name]), name
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("adjoint", [False, True])
def test_exact_operator_equals_the_oracle(gpu_lib, adjoint):
    rng = np.random.default_rng(5)
    o = oracle_case((12, 10, 9), adjoint=adjoint)
    for name in ("Vx", "Vy", "Vz", "Pt"):
        o.f[name][...] = rng.standard_normal(o.f[name].shape)
    if adjoint:  # the transposed system's ghosts are zero
        nx, ny, nz = 12, 10, 9
        for name, sl in (("Vx", (slice(None), [0, ny - 1], slice(None))), ("Vx", (slice(None), slice(None), [0, nz - 1])),
                         ("Vy", ([0, nx - 1], slice(None), slice(None))), ("Vy", (slice(None), slice(None), [0, nz - 1])),
                         ("Vz", ([0, nx - 1], slice(None), slice(None))), ("Vz", (slice(None), [0, ny - 1], slice(None)))):
            o.f[name][sl] = 0.0
    s = gpu_like(o, gpu_lib, adjoint)
    o.apply_operator()
    s.apply_operator()
    for name in ("txx", "tyy", "tzz", "txy", "txz", "tyz", "Rx", "Ry", "Rz", "divV"):
        assert np.array_equal(s.get(name), o.f[name]), name
    s.close()


@pytest.mark.gpu
def test_gradient_kernel_equals_the_oracle(gpu_lib):
    rng = np.random.default_rng(9)
    n = (13, 12, 10)
    fo, ao = oracle_case(n), oracle_case(n, adjoint=True)
    for o in (fo, ao):
        for name in ("Vx", "Vy", "Vz"):
            o.f[name][...] = rng.standard_normal(o.f[name].shape)
    fs, as_ = gpu_like(fo, gpu_lib), gpu_like(ao, gpu_lib, adjoint=True)
    fs.gradient_logmu(as_)
    assert np.array_equal(fs.get("grad"), fo.grad_logmu(ao))
    fs.close()
    as_.close()


@pytest.mark.gpu
@pytest.mark.parametrize("add", [False, True])
def test_visco_elastic_gradient_kernel_equals_the_oracle(gpu_lib, add):
    rng = np.random.default_rng(13)
    n = (13, 12, 10)
    fo, ao = oracle_case(n, variant="3d_ve_perf"), oracle_case(n, adjoint=True, variant="3d_ve_perf")
    for o in (fo, ao):
        for name in ITER_FIELDS[4:]:
            o.f[name][...] = rng.standard_normal(o.f[name].shape)
    fs = gpu_like(fo, gpu_lib, variant="3d_ve_perf")
    as_ = gpu_like(ao, gpu_lib, adjoint=True, variant="3d_ve_perf")
    g0 = rng.standard_normal((13, 12, 10))
    if add:
        fs.gradient_logmu(as_)  # allocates "grad"
        fs.set("grad", g0)
    fs.gradient_logmu(as_, add=add)
    ref = fo.grad_logmu_ve(ao, out=np.asfortranarray(g0.copy()) if add else None)
    assert np.array_equal(fs.get("grad"), ref)
    fs.close()
    as_.close()


@pytest.mark.gpu
def test_visco_elastic_gradient_matches_central_differences(gpu_lib):
    from ptstokes.adjoint import ViscoElasticAdjoint, inclusion_set, lognormal_factor, viscosity_field
    n = (18, 17, 16)
    incl = inclusion_set(seed=1855, log10_mu=(-2.0, 2.0))
    mus = viscosity_field(*n, incl)
    p = ViscoElasticAdjoint(*n, nt=3, lib=gpu_lib, eps=1e-12, nout=100, iter_max=1e6)
    p.set_viscosity(mus * lognormal_factor(n, seed=1856), nsmooth=10)
    p.forward()
    vobs = p.top_vz()
    p.set_inclusions(incl, nsmooth=10)  # the same field, built on the device
    J0, g, fo, ao = p.misfit_gradient(vobs)
    assert all(r["converged"] for r in fo + ao)
    mus0 = p.mus.copy()
    rng = np.random.default_rng(5)
    cand = np.argwhere(np.abs(g) >= 1e-3 * np.abs(g).max())
    cells = [tuple(c) for c in cand[rng.choice(len(cand), 12, replace=False)]]
    h = 1e-3
    worst = 0.0
    for c in cells:
        Js = []
        for sgn in (1, -1):
            m = mus0.copy()
            m[c] *= math.exp(sgn * h)
            p.mus = m
            p.forward()
            r = p.top_vz() - vobs
            Js.append(0.5 * float(np.sum(r * r)))
        fd = (Js[0] - Js[1]) / (2 * h)
        worst = max(worst, abs(g[c] - fd) / abs(fd))
    assert worst <= 1e-5, worst
    p.close()


@pytest.mark.gpu
def test_transposed_system_dot_product_on_the_gpu(gpu_lib):
    from ptstokes import Solver
    rng = np.random.default_rng(21)
    nx, ny, nz = 31, 29, 27
    fw = Solver("3d_v", nx, ny, nz, lib=gpu_lib).setup_inclusion(musi=1e-2)
    ad = Solver("3d_v", nx, ny, nz, lib=gpu_lib, adjoint=1)
    ad.init_inclusion(1.0, 1.0, 0.0, 0.0)
    ad.set("Mus", fw.get("Mus"))

    def interior(name, a):
        return {"Vx": a[1:nx, 1:ny - 1, 1:nz - 1], "Vy": a[1:nx - 1, 1:ny, 1:nz - 1],
                "Vz": a[1:nx - 1, 1:ny - 1, 1:nz], "Pt": a}[name]

    u, w = {}, {}
    for s, store, copies in ((fw, u, True), (ad, w, False)):
        for name in ("Vx", "Vy", "Vz", "Pt"):
            a = np.zeros(s.shape(name), order="F")
            v = interior(name, a)
            v[...] = rng.standard_normal(v.shape)
            s.set(name, a)
        if copies:
            s.apply_bc()
        for name in ("Vx", "Vy", "Vz", "Pt"):
            store[name] = interior(name, s.get(name)).copy()
    fw.apply_operator()
    ad.apply_operator()
    pairs = (("Rx", "Vx"), ("Ry", "Vy"), ("Rz", "Vz"), ("divV", "Pt"))
    lhs = sum(float(np.sum(fw.get(r) * w[v])) for r, v in pairs)
    rhs = sum(float(np.sum(u[v] * ad.get(r))) for r, v in pairs)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs), (lhs, rhs)
    fw.close()
    ad.close()


def _problem(gpu_lib, n, seed=1855):
    from ptstokes.adjoint import ViscousAdjoint, inclusion_set, lognormal_factor, viscosity_field
    incl = inclusion_set(seed=seed)
    mus = viscosity_field(*n, incl)
    p = ViscousAdjoint(*n, lib=gpu_lib, eps=1e-12, nout=100, iter_max=1e6)
    p.set_viscosity(mus * lognormal_factor(n, seed=seed + 1), nsmooth=10)
    p.forward()
    vobs = p.top_vz()
    # the field of the gradient is built on the device; the host path gives the same bits
    p.set_inclusions(incl, nsmooth=10)
    dev = p.mus.copy()
    p.set_viscosity(mus, nsmooth=10)
    assert np.array_equal(p.mus, dev)
    p.set_inclusions(incl, nsmooth=10)
    return p, vobs


@pytest.mark.gpu
def test_gradient_matches_central_differences_at_32_cells(gpu_lib):
    n = (24, 22, 20)
    p, vobs = _problem(gpu_lib, n)
    J0, g, fo, ao = p.misfit_gradient(vobs)
    assert fo["converged"] and ao["converged"]
    mus0 = p.mus.copy()
    rng = np.random.default_rng(32)
    # 32 random cells among those whose sensitivity is within 1e-3 of the largest (a cell far
    # from the observed plane changes J by less than the solver tolerance resolves)
    cand = np.argwhere(np.abs(g) >= 1e-3 * np.abs(g).max())
    cells = [tuple(c) for c in cand[rng.choice(len(cand), 32, replace=False)]]
    h = 1e-3
    worst = 0.0
    for c in cells:
        Js = []
        for sgn in (1, -1):
            m = mus0.copy()
            m[c] *= math.exp(sgn * h)
            p.set_viscosity(m, nsmooth=0)
            p.forward()
            r = p.top_vz() - vobs
            Js.append(0.5 * float(np.sum(r * r)))
        fd = (Js[0] - Js[1]) / (2 * h)
        worst = max(worst, abs(g[c] - fd) / abs(fd))
    assert worst <= 1e-5, worst
    p.close()


@pytest.mark.gpu
def test_torch_autograd_wrapper_gives_the_adjoint_gradient(gpu_lib):
    import torch
    from ptstokes.adjoint import top_vz
    n = (16, 15, 14)
    p, vobs = _problem(gpu_lib, n)
    logmu = torch.tensor(np.log(p.mus), dtype=torch.float64, device="cuda", requires_grad=True)
    v = top_vz(logmu, p)
    J = 0.5 * ((v - torch.from_numpy(vobs).cuda()) ** 2).sum()
    J.backward()
    J0, g, _, _ = p.misfit_gradient(vobs)
    assert abs(J.item() - J0) <= 1e-14 * J0
    assert np.array_equal(logmu.grad.cpu().numpy(), g)
    p.close()
