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
    """Cell (i,j,k) takes 10**log10_mu of the last sphere whose radius exceeds the distance of
    its centre ((i+1/2)dx, ...), else 1; the bounding-box shortcut must change nothing."""
    from ptstokes.adjoint import inclusion_set, viscosity_field
    n = (17, 13, 11)
    inc = inclusion_set(count=6, seed=3, radius=(1.0, 2.5))
    got = viscosity_field(*n, inc)
    h = [10.0 / m for m in n]
    x, y, z = [(np.arange(m) + 0.5) * d for m, d in zip(n, h)]
    want = np.ones(n)
    for q in inc:
        (cx, cy, cz), r = q["centre"], q["radius"]
        d2 = (x[:, None, None] - cx) ** 2 + (y[None, :, None] - cy) ** 2 + (z[None, None, :] - cz) ** 2
        want[d2 < r * r] = 10.0 ** q["log10_mu"]
    assert got.flags.f_contiguous and np.array_equal(got, want)


def test_lognormal_factor_has_the_requested_spread():
    from ptstokes.adjoint import lognormal_factor
    f = lognormal_factor((48, 40, 36), sigma=0.5, corr=4.0, seed=7)
    lg = np.log10(f)
    assert abs(lg.std() - 0.5) < 1e-9 and abs(lg.mean()) < 0.05
    # correlated: neighbouring cells are close, unlike white noise
    assert np.corrcoef(lg[:-1].ravel(), lg[1:].ravel())[0, 1] > 0.9
