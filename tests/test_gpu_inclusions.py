"""pts_init_inclusions (create_inclusions!, scripts/Stokes2D_param.jl:83-99) on the GPU: the
viscosity field of a list of inclusions is built on the device and equals the oracle's
restatement and the host generator bit for bit, in 2D (the reference's own case: one radius,
one inclusion viscosity) and in 3D (the 20-sphere field of the mixed-precision and adjoint
configurations, radii and viscosities per sphere, overlaps resolved by the first hit)."""
import ctypes

import numpy as np
import pytest

from oracle.binding import arr, lib as olib


def oracle_mus(shape, rows, d3, box=(10.0, 10.0, 10.0)):
    rows = np.ascontiguousarray(np.asarray(rows, dtype=np.float64).T)
    mus = np.zeros(shape if d3 else shape + (1,), order="F")
    ptr = [rows[q].ctypes.data_as(ctypes.c_void_p) for q in range(5)]
    h = [L / m for L, m in zip(box, shape)] + ([] if d3 else [1.0])
    olib().ora_create_inclusions_list(arr(mus), *ptr, rows.shape[1], 1.0, *h, box[0], box[1], box[2] if d3 else 1.0,
                                      1 if d3 else 0)
    return mus if d3 else mus[:, :, 0]


@pytest.mark.gpu
@pytest.mark.parametrize("variant,dims", [("3d_v", (47, 41, 37)), ("3d_ve_perf", (33, 35, 31)), ("3d_ve", (31, 29, 27))])
def test_sphere_list_field_bit_exact(gpu_lib, variant, dims):
    import ptstokes
    from ptstokes.adjoint import inclusion_array, inclusion_set, viscosity_field

    inc = inclusion_set(seed=1855, log10_mu=(-4.0, 4.0), radius=(0.6, 1.6))
    rows = inclusion_array(inc)
    s = ptstokes.Solver(variant, *dims, lib=gpu_lib)
    s.init_inclusions(rows, mus0=1.0, ebg=1.0)
    got = s.get("Mus")
    assert np.array_equal(got, oracle_mus(dims, rows, True))
    assert np.array_equal(got, viscosity_field(*dims, inc))
    assert len(np.unique(got)) >= 8  # many spheres hit
    # the velocities are the pure-shear ICs of the single-inclusion set-up, the rest zero
    r = ptstokes.Solver(variant, *dims, lib=gpu_lib)
    r.init_inclusion(1.0, 1e-3, 1.0, 1.0)
    for name in ("Vx", "Vy", "Vz", "Pt", "txx", "txy"):
        assert np.array_equal(s.get(name), r.get(name)), name
    s.close()
    r.close()


@pytest.mark.gpu
def test_reference_case_2d(gpu_lib):
    """Stokes2D_param.jl's form: circles of one radius and one inclusion viscosity, against the
    oracle's line-by-line restatement of create_inclusions! (ora2_create_inclusions)."""
    import ptstokes

    n = (63, 47)
    xs = np.array([-3.1, -1.0, 0.0, 1.2, 2.9, 0.4])
    ys = np.array([2.0, -2.5, 0.3, 1.1, -0.7, 3.3])
    r2, musi = 0.81, 1e-3
    rows = np.stack([xs, ys, np.zeros(6), np.full(6, r2), np.full(6, musi)], axis=1)
    s = ptstokes.Solver("2d_v", *n, lib=gpu_lib)
    s.init_inclusions(rows, mus0=1.0, ebg=1.0)
    want = np.zeros(n, order="F")
    rhog = np.zeros(n, order="F")
    olib().ora2_create_inclusions(arr(want), arr(rhog), xs.ctypes.data_as(ctypes.c_void_p),
                                  ys.ctypes.data_as(ctypes.c_void_p), len(xs), r2, 1.0, musi, 0.0, 1.0,
                                  10.0 / n[0], 10.0 / n[1], 10.0, 10.0)
    assert (want == musi).sum() > 20
    assert np.array_equal(s.get("Mus"), want)
    s.close()


@pytest.mark.gpu
def test_empty_list_and_rejections(gpu_lib):
    import ptstokes
    from ptstokes import _abi

    s = ptstokes.Solver("3d_v", 19, 17, 15, lib=gpu_lib)
    s.init_inclusions(np.zeros((0, 5)), mus0=2.5, ebg=1.0)
    assert np.all(s.get("Mus") == 2.5)
    bad = (_abi.PtsInclusion * 1)(_abi.PtsInclusion(0.0, float("nan"), 0.0, 1.0, 1.0))
    assert gpu_lib.pts_init_inclusions(s.ctx, bad, 1, 1.0, 1.0) == _abi.PTS_E_INVAL
    assert gpu_lib.pts_init_inclusions(s.ctx, bad, -1, 1.0, 1.0) == _abi.PTS_E_INVAL
    assert gpu_lib.pts_init_inclusions(s.ctx, None, 3, 1.0, 1.0) == _abi.PTS_E_INVAL
    s.close()
