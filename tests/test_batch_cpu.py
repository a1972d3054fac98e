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
