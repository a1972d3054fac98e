"""The aspect-ratio study on the GPU (ptstokes.scripts.Stokes2D_ve_param, aspect_ratio_sweep)
against the oracle's restatement of scripts/Stokes2D_ve_param.jl: the same iterations per
Maxwell step, every field bit for bit, the check's error to 1e-12 relative (its sums run in
another order); and the published totals of output/out_Stokes2D_ve_aspect_ratio_param.txt."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["Pt", "Vx", "Vy", "txx", "tyy", "txy", "Mus", "Must", "Gdt", "dtRho"]


def published():
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_output_lines.json")))
    return [r.split() for r in d["out_Stokes2D_ve_aspect_ratio_param.txt"]]


@pytest.mark.parametrize("ny,nsub,fact", [(31, 1, 1.0), (31, 2, 0.5), (63, 4, 0.3), (127, 1, 0.5), (127, 2, 0.4)])
def test_param_script_bit_exact(gpu_lib, ny, nsub, fact):
    from ptstokes.scripts import Stokes2D_ve_param
    from oracle import scripts as S

    o = S.VE2DParam(ny, nsub=nsub, fact=fact).setup().run()
    _, g, res = Stokes2D_ve_param(ny, nsub, fact, return_solver=True, lib=gpu_lib)
    assert res["iters"] == o.iters and res["ittot"] == o.ittot
    bad = [n for n in FIELDS if not np.array_equal(g.get(n), o.f[n])]
    assert not bad, bad
    err = o.err_hist[-1][2]
    assert abs(res["last"]["err"] - err) <= 1e-12 * err
    for a, b in zip((res["last"]["norm_Rx"], res["last"]["norm_Ry"], res["last"]["norm_divV"]), o.err_hist[-1][3]):
        assert abs(a - b) <= 1e-12 * abs(b)
    g.close()


def test_param_script_published_totals(gpu_lib):
    """Rows of the published sweep (ny = 127, nsub 1 and 2): the script's output line, up to
    the error's last digits, and the iteration total exactly."""
    from ptstokes.scripts import Stokes2D_ve_param

    for nx, ny, nsub, fact, ittot, nt, err in published():
        if ny != "127" or nsub not in ("1", "2") or fact not in ("1.0", "0.5", "0.1"):
            continue
        _, g, res = Stokes2D_ve_param(int(ny), int(nsub), float(fact), return_solver=True, lib=gpu_lib)
        got = res["line"].split()
        assert got[:6] == [nx, ny, nsub, fact, ittot, nt], (got, ittot)
        assert abs(float(got[6]) - float(err)) <= 1e-9 * float(err)
        g.close()


def test_sweep_runs_contexts_concurrently(gpu_lib):
    """aspect_ratio_sweep with three contexts in flight: every instance as the serial oracle."""
    from ptstokes.scripts import aspect_ratio_sweep
    from oracle import scripts as S

    out = aspect_ratio_sweep(facts=(1.0, 0.5), nsubs=(1, 2), resols=(31, 63), in_flight=3, lib=gpu_lib)
    assert len(out) == 8
    for r in out:
        o = S.VE2DParam(r["ny"], nsub=r["nsub"], fact=r["fact"]).setup().run()
        assert r["iters"] == o.iters, (r["ny"], r["nsub"], r["fact"])
        assert r["line"].split()[:6] == [str(o.nx), str(r["ny"]), str(r["nsub"]), str(r["fact"]), str(o.ittot), "5"]


def test_norm_scales_validated(gpu_lib):
    import ptstokes
    from ptstokes import _abi

    s = ptstokes.Solver("2d_ve", 31, 31, lib=gpu_lib)
    assert gpu_lib.pts_set_norm_scales(s.ctx, 0.0, 1.0, 1.0, 1.0) == _abi.PTS_E_INVAL
    assert gpu_lib.pts_set_norm_scales(s.ctx, 1.0, float("nan"), 1.0, 1.0) == _abi.PTS_E_INVAL
    assert gpu_lib.pts_set_norm_scales(s.ctx, 10.0, 10.0, 1.0, 10.0) == _abi.PTS_OK
    s.close()
