"""Host-side problem generators of the adjoint and mixed-precision configurations (no GPU)."""
import numpy as np


def test_inclusion_set_is_seeded_and_in_range():
    from ptstokes.adjoint import inclusion_set
    a = inclusion_set(seed=1855)
    assert a == inclusion_set(seed=1855) and a != inclusion_set(seed=1856)
    assert len(a) == 20
    for inc in a:
        assert all(0.0 <= c <= 10.0 for c in inc["centre"])
        assert 0.3 <= inc["radius"] <= 0.8 and -4.0 <= inc["log10_mu"] <= 4.0


def test_viscosity_field_matches_a_direct_evaluation():
    """create_inclusions! (Stokes2D_param.jl:83-99) in 3D, written as a plain loop: cell (i,j,k)
    takes 10**log10_mu of the FIRST sphere whose squared distance from its centre is below r2
    (centres in the centred frame x = (ix-1)*dx + 0.5*dx - 0.5*lx), else 1."""
    from ptstokes.adjoint import inclusion_array, inclusion_set, viscosity_field
    n = (17, 13, 11)
    inc = inclusion_set(count=6, seed=3, radius=(1.0, 2.5))
    got = viscosity_field(*n, inc)
    rows = inclusion_array(inc)
    h = [10.0 / m for m in n]
    want = np.ones(n)
    for i in range(n[0]):
        for j in range(n[1]):
            for k in range(n[2]):
                x, y, z = [(q * d + 0.5 * d) - 5.0 for q, d in zip((i, j, k), h)]
                for xi, yi, zi, r2, mu in rows:
                    if ((x - xi) * (x - xi) + (y - yi) * (y - yi)) + (z - zi) * (z - zi) < r2:
                        want[i, j, k] = mu
                        break
    overlapping = sum(1 for v in np.unique(got) if v != 1.0)
    assert overlapping >= 3  # several spheres (and their overlaps) are hit
    assert got.flags.f_contiguous and np.array_equal(got, want)


def test_viscosity_field_equals_the_oracle_restatement():
    """The host generator and the oracle's create_inclusions! restatement agree bit for bit,
    in 3D and (one z-plane, z term absent) in 2D, where the reference's own single-viscosity
    form (ora2_create_inclusions) agrees too."""
    import ctypes
    from oracle.binding import arr, lib
    from ptstokes.adjoint import inclusion_array, inclusion_set, viscosity_field
    n = (29, 23, 19)
    inc = inclusion_set(count=12, seed=11, radius=(0.8, 2.0))
    rows = np.ascontiguousarray(inclusion_array(inc).T)  # x, y, z, r2, mus as rows
    ptr = [rows[q].ctypes.data_as(ctypes.c_void_p) for q in range(5)]
    mus = np.zeros(n, order="F")
    lib().ora_create_inclusions_list(arr(mus), *ptr, rows.shape[1], 1.0, *(10.0 / m for m in n), 10.0, 10.0, 10.0, 1)
    assert np.array_equal(mus, viscosity_field(*n, inc))
    # 2D: the reference's case (one radius, one inclusion viscosity)
    n2 = (41, 37)
    xs = np.array([-2.0, 0.5, 1.75, 3.0]); ys = np.array([1.0, -0.5, 2.25, -3.0])
    r2, musi = 0.9, 1e-3
    a = np.zeros(n2, order="F"); rhog = np.zeros(n2, order="F")
    lib().ora2_create_inclusions(arr(a), arr(rhog), xs.ctypes.data_as(ctypes.c_void_p),
                                 ys.ctypes.data_as(ctypes.c_void_p), len(xs), r2, 1.0, musi, 0.0, 1.0,
                                 10.0 / n2[0], 10.0 / n2[1], 10.0, 10.0)
    b = np.zeros(n2 + (1,), order="F")
    zs, r2s, mus_i = np.zeros(4), np.full(4, r2), np.full(4, musi)
    lib().ora_create_inclusions_list(arr(b), xs.ctypes.data_as(ctypes.c_void_p), ys.ctypes.data_as(ctypes.c_void_p),
                                     zs.ctypes.data_as(ctypes.c_void_p), r2s.ctypes.data_as(ctypes.c_void_p),
                                     mus_i.ctypes.data_as(ctypes.c_void_p), 4, 1.0, 10.0 / n2[0], 10.0 / n2[1], 1.0,
                                     10.0, 10.0, 1.0, 0)
    assert (a == musi).sum() > 0 and np.array_equal(a, b[:, :, 0])


def test_lognormal_factor_has_the_requested_spread():
    from ptstokes.adjoint import lognormal_factor
    f = lognormal_factor((48, 40, 36), sigma=0.5, corr=4.0, seed=7)
    lg = np.log10(f)
    assert abs(lg.std() - 0.5) < 1e-9 and abs(lg.mean()) < 0.05
    # correlated: neighbouring cells are close, unlike white noise
    assert np.corrcoef(lg[:-1].ravel(), lg[1:].ravel())[0, 1] > 0.9
