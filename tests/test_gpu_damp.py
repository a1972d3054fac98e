"""The damped 2D variants (scripts/previous_damp/Stokes2D0.jl, Stokes2D_ve0.jl) on the GPU,
through the C ABI, against the CPU oracle: every field bit for bit, the check's norms to
1e-12 relative, iteration counts equal."""
import numpy as np
import pytest

from test_gpu_parity import assert_fields_equal, make_pair

pytestmark = pytest.mark.gpu

VARIANTS = ["2d_v_damp", "2d_ve_damp"]
DIMS = (47, 39)
ITERATED = ["Pt", "Vx", "Vy", "txx", "tyy", "txy", "dVx", "dVy"]


@pytest.mark.parametrize("variant", VARIANTS)
def test_setup_bit_exact(gpu_lib, variant):
    """ICs, smoothing, maxloc and compute_timesteps!."""
    o, g = make_pair(gpu_lib, variant, DIMS)
    assert_fields_equal(o, g, ["Vx", "Vy", "Mus", "Must", "dtVx", "dtVy", "dtPt"])
    g.close()


@pytest.mark.parametrize("variant", VARIANTS)
def test_iterations_bit_exact(gpu_lib, variant):
    """Two 'physical steps' of the fast path; the damped rates carry over between them."""
    o, g = make_pair(gpu_lib, variant, DIMS)
    for nit in (37, 23):
        if o.elastic:
            o.assign_tau()
            g.assign_tau()
        for _ in range(nit):
            o.iteration()
        g.iterate(nit)
        g.sync()
        assert_fields_equal(o, g, ITERATED)
    g.close()


@pytest.mark.parametrize("variant", VARIANTS)
def test_roles_and_check(gpu_lib, variant):
    """compute_P!, compute_τ!, compute_dV!, compute_V! and the bc calls one by one, then the
    check (Rx, Ry from compute_dV!, ∇V from compute_P!)."""
    o, g = make_pair(gpu_lib, variant, DIMS)
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
    assert_fields_equal(o, g, ITERATED + ["Rx", "Ry", "divV"])
    err_o, norms_o = o.check()
    chk = g.compute_res()
    np.testing.assert_allclose([chk["norm_Rx"], chk["norm_Ry"], chk["norm_divV"]], norms_o, rtol=1e-12)
    assert abs(chk["err"] - err_o) <= 1e-12 * err_o
    g.close()


@pytest.mark.parametrize("variant,dims", [("2d_v_damp", (47, 39)), ("2d_ve_damp", (31, 31)),
                                          ("2d_ve_damp", (127, 127))])
def test_full_run_bit_exact(gpu_lib, variant, dims):
    """The scripts' whole time loop and PT loop: same iterations per step, same fields."""
    o, g = make_pair(gpu_lib, variant, dims)
    o.run()
    res = g.run()
    assert res["iters"] == o.iters and res["converged"]
    assert_fields_equal(o, g, ITERATED)
    g.close()


def test_damping_numerics_are_used(gpu_lib):
    """Non-default Vdmp, β_n, Vsc, Ptsc through pts_set_damping (before compute_timesteps!)."""
    kw = dict(Vdmp=3.0, beta_n=1.0, Vsc=1.5, Ptsc=4.0)
    o, g = make_pair(gpu_lib, "2d_ve_damp", DIMS, **kw)
    assert_fields_equal(o, g, ["dtVx", "dtVy", "dtPt"])
    o.assign_tau()
    g.assign_tau()
    for _ in range(29):
        o.iteration()
    g.iterate(29)
    g.sync()
    assert_fields_equal(o, g, ITERATED)
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
