"""The batched visco-elastic aspect-ratio sweep (ptstokes.batch.BatchVE, one persistent
launch for every instance of scripts/runme_Stokes2D_aspect_ratio.jl) against the oracle's
restatement of scripts/Stokes2D_ve_param.jl run instance by instance: the same iterations in
every Maxwell step, every field bit for bit, the check's error to 1e-12 relative (its sums run
in another order); and the published totals of output/out_Stokes2D_ve_aspect_ratio_param.txt
from one launch."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["Pt", "Vx", "Vy", "txx", "tyy", "txy", "txx_o", "tyy_o", "txy_o", "Mus", "Must", "Gdt", "dtRho", "divV",
          "Rx", "Ry"]
# uneven instances: nx = nsub*(ny+1)-1 of 31, 63, 71 and 47 cells, so each checks on its own cadence
CASES = [dict(ny=31, nsub=1, fact=1.0), dict(ny=31, nsub=2, fact=0.5), dict(ny=23, nsub=3, fact=0.3),
         dict(ny=47, nsub=1, fact=0.7)]


def _compare(b, res, q, o):
    assert res["steps"][q] == o.iters, (q, res["steps"][q], o.iters)
    assert res["ittot"][q] == o.ittot
    bad = [n for n in FIELDS if not np.array_equal(b.get(q, n), o.f[n])]
    assert not bad, (q, bad)
    if o.err_hist:
        err = o.err_hist[-1][2]
        assert abs(res["err"][q] - err) <= 1e-12 * err
    else:  # no check in its steps: err stays the 2ε each step starts with
        assert res["err"][q] == 2 * 1e-6


@pytest.mark.parametrize("tile", [1, 2])
def test_batch_ve_equals_the_oracle_per_instance(gpu_lib, tile):
    from ptstokes.batch import BatchVE
    from oracle import scripts as S

    b = BatchVE(CASES, tile=tile, lib=gpu_lib)
    b.setup()
    res = b.solve()
    assert res["used_graph"] and not res["nan"]
    assert all(res["converged"])
    for q, d in enumerate(CASES):
        o = S.VE2DParam(d["ny"], nsub=d["nsub"], fact=d["fact"]).setup().run()
        _compare(b, res, q, o)
    b.close()


def test_batch_ve_steps_stopped_by_iter_max(gpu_lib):
    """A common iterMax of 40 (41 iterations per step, past the first check of the nx = 31
    instance; the nx = 63 one never checks) on 3 and 2 steps: the unconverged steps end on
    iterMax, assign_τ! runs between them, and every field equals the oracle's run with the
    same limit."""
    from ptstokes.batch import BatchVE
    from oracle import scripts as S

    lib = gpu_lib
    cases = [dict(CASES[0], nt=3), dict(CASES[1], nt=2)]
    b = BatchVE(cases, iter_max=40, lib=lib)
    b.setup()
    res = b.solve()
    assert res["steps"] == [[41, 41, 41], [41, 41]]
    assert res["converged"] == [False, False]
    for q, d in enumerate(cases):
        o = S.VE2DParam(d["ny"], nsub=d["nsub"], fact=d["fact"]).setup().run(nt=d["nt"], iter_max=40)
        _compare(b, res, q, o)
    b.close()


def test_batch_ve_runs_again_after_setup(gpu_lib):
    from ptstokes.batch import BatchVE

    b = BatchVE(CASES[:2], lib=gpu_lib)
    b.setup()
    r1 = b.solve()
    p1 = b.get(1, "Pt")
    b.setup()
    r2 = b.solve()
    assert r1["steps"] == r2["steps"] and r1["err"] == r2["err"]
    assert np.array_equal(p1, b.get(1, "Pt"))
    b.close()


def test_batch_ve_published_totals_in_one_launch(gpu_lib):
    """The published rows with ny = 127 and nsub 1 and 2 (20 instances) as one batch: every
    instance's output line, the error up to its last digits, the iteration total exactly."""
    from ptstokes.batch import BatchVE

    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_output_lines.json")))
    rows = [r.split() for r in d["out_Stokes2D_ve_aspect_ratio_param.txt"]]
    rows = [r for r in rows if r[1] == "127" and r[2] in ("1", "2")]
    assert len(rows) == 20
    b = BatchVE([dict(ny=int(r[1]), nsub=int(r[2]), fact=float(r[3])) for r in rows], lib=gpu_lib)
    b.setup()
    res = b.solve()
    for q, (nx, ny, nsub, fact, ittot, nt, err) in enumerate(rows):
        got = res["lines"][q].split()
        assert got[:6] == [nx, ny, nsub, fact, ittot, nt], (got, ittot)
        assert abs(float(got[6]) - float(err)) <= 1e-9 * float(err)
    b.close()


def test_autotune_picks_a_tile_for_the_ve_sweep(gpu_lib, tmp_path, monkeypatch):
    """The autotuner times the four tile shapes on a visco-elastic batch (two checks of its
    smallest instance), caches the choice under a key of its own, and the sweep run on the
    chosen tile still equals the oracle."""
    from ptstokes.batch import TILE_SHAPES, BatchVE, _batch_key, autotune
    from oracle import scripts as S

    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    b = BatchVE(CASES[:2], lib=gpu_lib)
    b.setup()
    entry = autotune(b)
    assert entry["iters"] == 2 * 31 - 1 and len(entry["ms"]) == len(TILE_SHAPES)
    assert b.tile == entry["tile"] and _batch_key(b).startswith("2d|ve|")
    assert autotune(b)["tile"] == entry["tile"]  # from the cache
    res = b.solve()
    for q, d in enumerate(CASES[:2]):
        o = S.VE2DParam(d["ny"], nsub=d["nsub"], fact=d["fact"]).setup().run()
        _compare(b, res, q, o)
    b.close()
