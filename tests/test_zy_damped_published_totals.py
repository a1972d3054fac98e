"""The damped visco-elastic script (scripts/previous_damp/Stokes2D_ve0.jl) on the GPU, checked
with the error measure the script keeps commented out beside its check (:166,
norm(R)/length(R)), the measure the reference's output/out_Stokes2D_ve0.txt was written
with: ptstokes.scripts.Stokes2D_ve0(err_form="length") must take the published iteration
totals, with the same per-step counts as the oracle's run with that measure.

The step loop runs from the host through the context's assign_tau, iterate and compute_res.
Each of those is compared with the oracle in tests/test_gpu_damp.py, and the loop itself is
checked on the CPU in tests/test_damp_driver_cpu.py. This file puts the three together on a
B200. Its name sorts it after the other GPU tests.
"""
import json
import os

import pytest

from conftest import GOLDEN


@pytest.mark.gpu
@pytest.mark.parametrize("n", [31, 63])
def test_gpu_takes_the_published_damped_totals(gpu_lib, n):
    import ptstokes
    from oracle import scripts as S

    with open(os.path.join(GOLDEN, "reference_output_lines.json")) as fh:
        lines = json.load(fh)["out_Stokes2D_ve0.txt"]
    published = {int(l.split()[0]): (int(l.split()[2]), int(l.split()[3])) for l in lines}
    (_, _, Pt), s, res = ptstokes.scripts.Stokes2D_ve0(n, n, return_solver=True, err_form="length", lib=gpu_lib)
    assert (res["ittot"], len(res["iters"])) == published[n]
    o = S.make("2d_ve_damp", n, n, err_form="length").run()
    assert res["iters"] == o.iters
    assert res["converged"]
    s.close()
