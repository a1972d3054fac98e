"""Host-side logic of the batched sweep: the seeded instance generator (no GPU)."""
import numpy as np


def test_sweep_instances_are_seeded_and_in_range():
    from ptstokes.batch import sweep_instances
    a = sweep_instances(256, seed=1855)
    b = sweep_instances(256, seed=1855)
    assert a == b and len(a) == 256
    assert {d["nx"] for d in a} <= {63, 127, 255, 511}
    for d in a:
        assert 1.0 <= d["lx"] / d["ly"] <= 4.0
        assert 1e-6 <= d["musi"] <= 1e-1
        assert (d["rhogi"], d["ebg"]) in ((1.0, 0.0), (0.0, 1.0))
        assert abs(d["lx"] / d["nx"] - d["ly"] / d["ny"]) < 0.25 * d["ly"] / d["ny"]
    frac = np.mean([d["rhogi"] for d in a])
    assert 0.35 < frac < 0.65


def test_batch_ve_create_rejects_bad_instances():
    """pts_batch_create_ve checks every instance before any CUDA call (runs without a GPU)."""
    import ctypes

    import ptstokes
    from ptstokes import _abi

    lib = ptstokes.load()
    desc = _abi.PtsBatchDesc()
    desc.tile, desc.eps, desc.r, desc.Re, desc.CFL = 1, 1e-6, 1.0, 15.7, 0.6
    bad = [dict(ny=2, nsub=1, nt=5, fact=1.0), dict(ny=31, nsub=0, nt=5, fact=1.0),
           dict(ny=31, nsub=1, nt=0, fact=1.0), dict(ny=31, nsub=1, nt=65, fact=1.0),
           dict(ny=31, nsub=1, nt=5, fact=0.0), dict(ny=31, nsub=1, nt=5, fact=1.0, musi=float("nan"))]
    for d in bad:
        inst = _abi.PtsBatchVEInstance(d["ny"], d["nsub"], d["nt"], 0, d["fact"], 10.0, d.get("musi", 1e-3))
        h = ctypes.c_void_p()
        assert lib.pts_batch_create_ve(ctypes.byref(desc), ctypes.byref(inst), 1, ctypes.byref(h)) == _abi.PTS_E_INVAL
        assert not h.value
    h = ctypes.c_void_p()
    inst = _abi.PtsBatchVEInstance(31, 1, 5, 0, 1.0, 10.0, 1e-3)
    desc.CFL = 0.0
    assert lib.pts_batch_create_ve(ctypes.byref(desc), ctypes.byref(inst), 1, ctypes.byref(h)) == _abi.PTS_E_INVAL


def test_aspect_ratio_instances_follow_the_driver_loop_order():
    """runme_Stokes2D_aspect_ratio.jl iterates Iterators.product(FACT, NSUB, RESOL): FACT fastest."""
    from ptstokes.batch import aspect_ratio_instances

    inst = aspect_ratio_instances(nsubs=(1, 2), resols=(127,))
    assert [(d["nsub"], d["fact"]) for d in inst[:11]] == [(1, f) for f in
                                                            (1.0, 0.9, 0.8, 0.7, 0.6, 0.5, 0.4, 0.3, 0.2, 0.1)] + [(2, 1.0)]
    assert len(inst) == 20 and all(d["ny"] == 127 and d["nt"] == 5 for d in inst)
