"""The host-driven step loop of the damped 2D scripts with their commented-out error
measure (ptstokes.scripts.run_length_error, length_error), checked on the CPU.

The loop only calls a context's assign_tau, iterate and compute_res, whose GPU results the
-m gpu tests compare with the oracle (tests/test_gpu_damp.py). Here the oracle stands in for
the context: `OracleContext` answers the same calls, with compute_res returning the check in
the form pts_compute_res gives it (norms scaled by the pressure or velocity range, lx and
1/sqrt(length)). The loop must then take the reference's published iteration totals
(output/out_Stokes2D_ve0.txt) and the same per-step counts as the oracle's own run with
the alternative measure (Stokes2D_ve0.jl:166).
"""
import json
import math
import os

import pytest

from conftest import GOLDEN


class OracleContext:
    """The calls run_length_error makes on a Solver, answered by the oracle's restatement."""

    def __init__(self, variant, n):
        from oracle import scripts as S

        self.o = S.make(variant, n, n)
        self.o.setup()
        self.variant, self.ndim, self.nx, self.ny = variant, 2, n, n
        d = {"2d_ve_damp": dict(nt=5, nout=200, iter_max=2e5), "2d_v_damp": dict(nt=1, nout=500, iter_max=1e5)}
        self.p = dict(lx=10.0, eps=1e-8, **d[variant])
        self.calls = []

    def assign_tau(self):
        self.calls.append("assign_tau")
        self.o.assign_tau()

    def iterate(self, k):
        self.calls.append(k)
        for _ in range(k):
            self.o.iteration()

    def compute_res(self):
        from oracle.binding import stats

        f, lx = self.o.f, self.p["lx"]
        _, vmin, vmax = stats(f["Vx"])
        _, pmin, pmax = stats(f["Pt"])

        def scaled(name, rng):
            s, _, _ = stats(f[name])
            return math.sqrt(s) / rng * lx / math.sqrt(f[name].size)

        return dict(norm_Rx=scaled("Rx", pmax - pmin), norm_Ry=scaled("Ry", pmax - pmin),
                    norm_divV=scaled("divV", vmax - vmin), Vmin=vmin, Vmax=vmax, Pmin=pmin, Pmax=pmax)


def _published():
    with open(os.path.join(GOLDEN, "reference_output_lines.json")) as fh:
        lines = json.load(fh)["out_Stokes2D_ve0.txt"]
    return {int(l.split()[0]): (int(l.split()[2]), int(l.split()[3])) for l in lines}


@pytest.mark.parametrize("n", [31, 63])
def test_host_loop_takes_the_published_totals(n):
    from oracle import scripts as S
    from ptstokes.scripts import run_length_error

    ctx = OracleContext("2d_ve_damp", n)
    res = run_length_error(ctx)
    assert (res["ittot"], len(res["iters"])) == _published()[n]
    assert res["converged"] and res["err"] <= 1e-8
    ref = S.make("2d_ve_damp", n, n, err_form="length").run()
    assert res["iters"] == ref.iters
    # one assign_τ! per step, and blocks of PT iterations that end on the checks
    assert ctx.calls.count("assign_tau") == 5
    assert all(k == 200 for k in ctx.calls if k != "assign_tau")


def test_length_error_recovers_the_unscaled_norms():
    from oracle import scripts as S
    from ptstokes.scripts import length_error

    ctx = OracleContext("2d_ve_damp", 31)
    ctx.assign_tau()
    ctx.iterate(37)
    got, norms = length_error(ctx, ctx.compute_res())
    o = ctx.o
    assert isinstance(o, S.VE2DDamp)
    o.err_form = "length"  # the oracle's own form of the same measure
    want, want_norms = o.check()
    for a, b in zip(norms, want_norms):
        assert abs(a - b) <= 1e-13 * abs(b)
    assert abs(got - want) <= 1e-13 * want


def test_iter_max_ends_a_step_after_one_more_iteration():
    """`while err > ε && iter <= iterMax`: with iterMax = 250 and nout = 200 a step that does
    not converge runs 251 iterations, checked once at 200."""
    from ptstokes.scripts import run_length_error

    ctx = OracleContext("2d_ve_damp", 31)
    ctx.p.update(nt=2, iter_max=250)
    res = run_length_error(ctx)
    assert res["iters"] == [251, 251]
    assert [k for k in ctx.calls if k != "assign_tau"] == [200, 51, 200, 51]
    assert not res["converged"]


def test_err_form_is_validated_before_any_context_exists():
    from ptstokes import scripts

    with pytest.raises(ValueError):
        scripts.Stokes2D_ve0(31, 31, err_form="sqrt")
    with pytest.raises(ValueError):
        scripts.Stokes2D_ve(31, 31, err_form="length")


def test_length_error_refuses_a_3d_context():
    from ptstokes.scripts import length_error

    ctx = OracleContext("2d_ve_damp", 31)
    ctx.ndim = 3
    with pytest.raises(ValueError):
        length_error(ctx, {})


def test_host_loop_needs_a_check_cadence():
    from ptstokes.scripts import run_length_error

    ctx = OracleContext("2d_ve_damp", 31)
    ctx.p["nout"] = 0
    with pytest.raises(ValueError):
        run_length_error(ctx)
