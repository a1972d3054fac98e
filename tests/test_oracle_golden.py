"""The CPU oracle against the reference's own regression fixtures (test/reftest-files).

Each fixture pins the pressure Pt (sampled 12 points per dimension) and the cell
centres xc of one reference script run on the CPU Threads backend. The oracle must
reproduce them within Julia's `isapprox` (the reference's own comparison,
test/test_2D.jl:14); it in fact reproduces them bit for bit, which is asserted too.
"""
import json
import os

import numpy as np
import pytest

from conftest import julia_isapprox, load_golden

FIXTURES = [
    "test_Stokes_2D_v",
    "test_Stokes_2D_ve",
    "test_Stokes_2D_ve_perf",
    "test_Stokes3D_ve_multixpu",
    "test_Stokes3D_ve_multixpu_perf",
    "test_Stokes3D_ve_perf",
]


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_reproduces_reference_fixture(name):
    from oracle import scripts as S
    meta, P, X = load_golden(name)
    case = S.make(meta["variant"], *meta["grid"]).run()
    x, p = S.fixture_sample(case)
    assert p.shape == P.shape
    assert julia_isapprox(p, P) and julia_isapprox(x, X)
    # bit-exact: same kernels, same operation order, no FMA contraction
    assert np.array_equal(p, P)
    assert np.array_equal(x, X)


def test_oracle_iteration_counts_fixed():
    """The perf scripts run `iterMax+1` iterations (loop `iter <= iterMax`, nout > iterMax)."""
    from oracle import scripts as S
    assert S.make("2d_ve_perf", 15, 15).run().iters == [101]
    assert S.make("3d_ve_perf", 9, 9, 9).run().iters == [201]


def test_oracle_nan_raises():
    """A poisoned field makes the check's err NaN, which the scripts turn into error("NaN")."""
    from oracle import scripts as S
    c = S.make("2d_ve", 15, 15, nout=10)
    c.f["Pt"][3, 3] = np.nan
    with pytest.raises(FloatingPointError):
        c.run(nt=1)


def _published(name):
    """Rows of one of the reference's output files (tests/golden/reference_output_lines.json)."""
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_output_lines.json")))
    return [list(map(int, r.split()[:4])) for r in d[name]]


def test_oracle_reproduces_the_published_2d_ve_iteration_counts():
    """scripts/Stokes2D_ve.jl run to 1e-8 over 5 steps: output/out_Stokes2D_ve.txt lists the total
    iteration count per grid; the oracle takes exactly as many."""
    from oracle import scripts as S
    for nx, ny, ittot, nt in _published("out_Stokes2D_ve.txt"):
        if nx > 127:
            continue
        o = S.make("2d_ve", nx, ny)
        o.run()
        assert len(o.iters) == nt and sum(o.iters) == ittot, (nx, o.iters, ittot)


def test_oracle_reproduces_the_published_aspect_ratio_counts():
    """scripts/Stokes2D_ve_param.jl, as runme_Stokes2D_aspect_ratio.jl sweeps it:
    output/out_Stokes2D_ve_aspect_ratio_param.txt lists `nx ny nsub fact ittot nt err` per
    instance; the oracle takes exactly as many iterations (all ten facts of the 127^2 grid, two
    of the 255x127 grid with two inclusions) and ends at the same error."""
    from oracle import scripts as S
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_output_lines.json")))
    rows = [r.split() for r in d["out_Stokes2D_ve_aspect_ratio_param.txt"]]
    picked = [r for r in rows if r[:3] == ["127", "127", "1"]]
    picked += [r for r in rows if r[:3] == ["255", "127", "2"] and r[3] in ("0.5", "0.4")]
    assert len(picked) == 12
    for nx, ny, nsub, fact, ittot, nt, err in picked:
        o = S.VE2DParam(int(ny), nsub=int(nsub), fact=float(fact)).setup().run()
        assert o.nx == int(nx) and len(o.iters) == int(nt) and o.ittot == int(ittot), (nx, nsub, fact, o.iters)
        assert abs(o.err_hist[-1][2] - float(err)) <= 1e-9 * float(err), (nx, nsub, fact, o.err_hist[-1][2], err)
