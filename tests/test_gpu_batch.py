"""Batched 2D viscous sweep (one persistent cooperative launch) against the oracle.

Each instance of the batch must equal, bit for bit, the oracle's single-instance run of
the same problem (oracle.scripts.V2DSweep): the same iteration count to tolerance and
the same fields. The tile shape chosen by the autotuner must not change any result.
Instances that do not converge stop at their own iterMax inside the shared launch, and a
NaN in one instance freezes that instance only.
"""
import numpy as np
import pytest

CASES = [
    dict(nx=31, ny=31, lx=10.0, ly=10.0, musi=1e-3, radius2=1.0, rhogi=0.0, ebg=1.0),
    dict(nx=63, ny=31, lx=20.0, ly=10.0, musi=1e-4, radius2=1.0, rhogi=1.0, ebg=0.0),
    dict(nx=47, ny=23, lx=20.0, ly=10.0, musi=1e-6, radius2=1.0, rhogi=1.0, ebg=0.0),
    dict(nx=95, ny=31, lx=30.0, ly=10.0, musi=1e-2, radius2=1.0, rhogi=0.0, ebg=1.0),
    dict(nx=37, ny=37, lx=10.0, ly=10.0, musi=1e-5, radius2=1.0, rhogi=0.0, ebg=1.0),
]
FIELDS = ["Pt", "Vx", "Vy", "txx", "tyy", "txy", "Mus", "Must", "rhog"]


def oracle_case(d, **kw):
    from oracle import scripts as S
    return S.V2DSweep(d["nx"], d["ny"], lx=d["lx"], ly=d["ly"], musi=d["musi"], rhogi=d["rhogi"], ebg=d["ebg"],
                      **kw).setup()


@pytest.mark.gpu
def test_batch_equals_the_oracle_instance_by_instance(gpu_lib):
    from ptstokes.batch import Batch
    b = Batch(CASES, nout=100, eps=1e-8, iter_max=2e5, lib=gpu_lib).setup()
    res = b.solve()
    for q, d in enumerate(CASES):
        o = oracle_case(d, nout=100, iterMax=2e5).run()
        assert res["converged"][q]
        assert res["iters"][q] == o.iters[0], (q, res["iters"][q], o.iters)
        for name in FIELDS:
            assert np.array_equal(b.get(q, name), o.f[name]), (q, name)
    b.close()


@pytest.mark.gpu
def test_batch_tile_shapes_give_identical_results(gpu_lib):
    from ptstokes.batch import Batch, TILE_SHAPES
    ref = None
    for t in range(len(TILE_SHAPES)):
        b = Batch(CASES, nout=50, eps=1e-8, iter_max=2e5, tile=t, lib=gpu_lib).setup()
        res = b.solve(iter_limit=173)
        assert res["iters"] == [174] * len(CASES)
        got = [b.get(q, "Vy") for q in range(len(CASES))]
        if ref is None:
            ref = got
        else:
            assert all(np.array_equal(a, r) for a, r in zip(got, ref)), t
        b.close()


@pytest.mark.gpu
def test_batch_autotune_and_iter_limit(gpu_lib, tmp_path, monkeypatch):
    from ptstokes.batch import Batch, autotune
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    b = Batch(CASES, nout=100, eps=1e-8, iter_max=2e5, lib=gpu_lib).setup()
    entry = autotune(b, iters=150)
    assert entry["tile"] in range(4) and len(entry["ms"]) == 4
    again = autotune(b)  # served from the cache
    assert again["tile"] == entry["tile"]
    res = b.solve(iter_limit=150)
    o = oracle_case(CASES[2], nout=100, iterMax=150).run()
    assert res["iters"][2] == o.iters[0] == 151
    assert np.array_equal(b.get(2, "Pt"), o.f["Pt"])
    b.close()


@pytest.mark.gpu
def test_batch_each_instance_stops_at_its_own_iter_max(gpu_lib):
    """eps = 1e-300 is never reached: every instance runs to iterMax = 100max(nx,ny)
    (Stokes2D_param.jl:146), i.e. 100max(nx,ny) + 1 iterations, all in one launch."""
    from ptstokes.batch import Batch
    cases = [dict(nx=15, ny=11, lx=13.6, ly=10.0, musi=1e-3, radius2=1.0, rhogi=0.0, ebg=1.0),
             dict(nx=23, ny=17, lx=13.5, ly=10.0, musi=1e-5, radius2=1.0, rhogi=1.0, ebg=0.0),
             dict(nx=31, ny=9, lx=34.0, ly=10.0, musi=1e-2, radius2=1.0, rhogi=1.0, ebg=0.0)]
    b = Batch(cases, nout=100, eps=1e-300, iter_max=0, lib=gpu_lib).setup()
    res = b.solve()
    assert res["iters"] == [1501, 2301, 3101] and not any(res["converged"])
    for q, d in enumerate(cases):
        o = oracle_case(d, nout=100, eps=1e-300).run()
        assert o.iters[0] == res["iters"][q]
        for name in ("Pt", "Vx", "Vy", "txy"):
            assert np.array_equal(b.get(q, name), o.f[name]), (q, name)
    b.close()


@pytest.mark.gpu
def test_batch_nan_freezes_only_its_instance(gpu_lib):
    """A NaN density in one instance makes its check NaN: that instance is frozen and
    reported as not converged, the call reports PTS_E_NAN, the other instance converges
    exactly as it does alone."""
    from ptstokes import PtsError
    from ptstokes.batch import Batch
    good = CASES[1]
    bad = dict(good, rhogi=float("nan"))
    b = Batch([good, bad], nout=100, eps=1e-8, iter_max=2e5, lib=gpu_lib).setup()
    res = b.solve(raise_on_nan=False)
    assert res["nan"] and res["converged"] == [True, False] and res["iters"][1] == 100
    o = oracle_case(good, nout=100, iterMax=2e5).run()
    assert res["iters"][0] == o.iters[0]
    assert np.array_equal(b.get(0, "Vy"), o.f["Vy"])
    b.setup()
    with pytest.raises(PtsError):
        b.solve()
    b.close()
