"""The damped variants (scripts/previous_damp/Stokes2D0.jl, Stokes2D_ve0.jl and
scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl on one rank) on the GPU, through the
C ABI, against the CPU oracle: every field bit for bit, the check's norms to 1e-12
relative, iteration counts equal."""
import numpy as np
import pytest

from test_gpu_parity import assert_fields_equal, make_pair

pytestmark = pytest.mark.gpu

VARIANTS = ["2d_v_damp", "2d_ve_damp", "3d_v_damp"]
DIMS = {"2d_v_damp": (47, 39), "2d_ve_damp": (47, 39), "3d_v_damp": (35, 31, 33)}
ITERATED2 = ["Pt", "Vx", "Vy", "txx", "tyy", "txy", "dVx", "dVy"]
ITERATED3 = ["Pt", "Vx", "Vy", "Vz", "txx", "tyy", "tzz", "txy", "txz", "tyz", "dVx", "dVy", "dVz"]


def iterated(variant):
    return ITERATED3 if variant.startswith("3d") else ITERATED2


@pytest.mark.parametrize("variant", VARIANTS)
def test_setup_bit_exact(gpu_lib, variant):
    """ICs, smoothing, maxloc and compute_timesteps!."""
    o, g = make_pair(gpu_lib, variant, DIMS[variant])
    names = ["Vx", "Vy", "Mus", "Must", "dtVx", "dtVy", "dtPt"]
    if variant.startswith("3d"):
        names += ["Vz", "dtVz"]
    assert_fields_equal(o, g, names)
    g.close()


@pytest.mark.parametrize("variant", VARIANTS)
def test_iterations_bit_exact(gpu_lib, variant):
    """Two 'physical steps' of the fast path; the damped rates carry over between them."""
    o, g = make_pair(gpu_lib, variant, DIMS[variant])
    for nit in (37, 23):
        if o.elastic:
            o.assign_tau()
            g.assign_tau()
        for _ in range(nit):
            o.iteration()
        g.iterate(nit)
        g.sync()
        assert_fields_equal(o, g, iterated(variant))
    g.close()


@pytest.mark.parametrize("variant", VARIANTS)
def test_roles_and_check(gpu_lib, variant):
    """compute_P!, compute_τ!, compute_dV!, compute_V! and the bc calls one by one, then the
    check (R from compute_dV!, ∇V from compute_P!)."""
    o, g = make_pair(gpu_lib, variant, DIMS[variant])
    if o.elastic:
        o.assign_tau()
        g.assign_tau()
    for _ in range(13):
        o.iteration()
        g.compute_P()
        g.compute_tau()
        g.compute_dV()
        g.compute_V()
        g.apply_bc()
    g.sync()
    d3 = variant.startswith("3d")
    assert_fields_equal(o, g, iterated(variant) + ["Rx", "Ry", "divV"] + (["Rz"] if d3 else []))
    err_o, norms_o = o.check()
    chk = g.compute_res()
    got = [chk["norm_Rx"], chk["norm_Ry"]] + ([chk["norm_Rz"]] if d3 else []) + [chk["norm_divV"]]
    np.testing.assert_allclose(got, norms_o, rtol=1e-12)
    assert abs(chk["err"] - err_o) <= 1e-12 * err_o
    g.close()


@pytest.mark.parametrize("variant,dims", [("2d_v_damp", (47, 39)), ("2d_ve_damp", (31, 31)),
                                          ("2d_ve_damp", (127, 127)), ("3d_v_damp", (31, 31, 31))])
def test_full_run_bit_exact(gpu_lib, variant, dims):
    """The scripts' whole time loop and PT loop: same iterations per step, same fields."""
    o, g = make_pair(gpu_lib, variant, dims)
    o.run()
    res = g.run()
    assert res["iters"] == o.iters and res["converged"]
    assert_fields_equal(o, g, iterated(variant))
    g.close()


@pytest.mark.parametrize("variant", ["2d_ve_damp", "3d_v_damp"])
def test_damping_numerics_are_used(gpu_lib, variant):
    """Non-default Vdmp, β_n, Vsc, Ptsc through pts_set_damping (before compute_timesteps!)."""
    kw = dict(Vdmp=3.0, beta_n=1.0, Vsc=1.5, Ptsc=4.0)
    o, g = make_pair(gpu_lib, variant, DIMS[variant], **kw)
    assert_fields_equal(o, g, ["dtVx", "dtVy", "dtPt"] + (["dtVz"] if variant.startswith("3d") else []))
    if o.elastic:
        o.assign_tau()
        g.assign_tau()
    for _ in range(29):
        o.iteration()
    g.iterate(29)
    g.sync()
    assert_fields_equal(o, g, iterated(variant))
    g.close()


def test_set_damping_is_refused_for_other_variants(gpu_lib):
    import ptstokes
    s = ptstokes.Solver("2d_ve", 15, 15, lib=gpu_lib)
    with pytest.raises(ptstokes.PtsError):
        s.set_damping()
    s.close()
    s = ptstokes.Solver("2d_v_damp", 15, 15, lib=gpu_lib)
    with pytest.raises(ptstokes.PtsError):
        s.set_damping(Vsc=0.0)
    s.close()


def test_script_mirror(gpu_lib):
    """ptstokes.scripts.Stokes2D_ve0 returns (xc, yc, Pt) of the restated script."""
    import ptstokes
    from oracle import scripts as S
    o = S.make("2d_ve_damp", 63, 63).run()
    (xc, yc, Pt), s, res = ptstokes.scripts.Stokes2D_ve0(63, 63, return_solver=True)
    assert res["iters"] == o.iters
    assert np.array_equal(Pt, o.f["Pt"]) and np.array_equal(xc, o.xc)
    s.close()


def test_script_mirror_3d(gpu_lib):
    """ptstokes.scripts.Stokes3D0 returns (xc, yc, zc, Pt) of the restated one-rank script."""
    import ptstokes
    from oracle import scripts as S
    o = S.make("3d_v_damp", 31, 33, 35).run()
    (xc, yc, zc, Pt), s, res = ptstokes.scripts.Stokes3D0(31, 33, 35, return_solver=True)
    assert res["iters"] == o.iters
    assert np.array_equal(Pt, o.f["Pt"])
    s.close()
