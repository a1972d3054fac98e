"""Mixed precision (FP32 inner PT sweeps on a correction, FP64 defect correction) on the GPU.

The reference has no mixed-precision mode, so parity is stated against the FP64 path:
the oracle (CPU, bit-identical to the reference's Float64 arithmetic) and the plain FP64
GPU path. The bar: converged fields within 1e-6 relative (L2 per field) of the FP64
oracle, the same iteration count to tolerance up to one check interval, and the FP64
check of the final iterate below the tolerance.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F3 = ["Pt", "Vx", "Vy", "Vz", "txx", "tyy", "tzz", "txy", "txz", "tyz"]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("variant,dims,nt", [("3d_ve_perf", (23, 21, 19), 2), ("3d_v", (21, 19, 23), 1)])
def test_mixed_converges_to_the_fp64_solution(gpu_lib, variant, dims, nt):
    import ptstokes
    from oracle import scripts as S

    kw = dict(nout=100, nt=nt, iter_max=2e5, eps=1e-8)
    o = S.make(variant, *dims, nout=100, nt=nt, iterMax=2e5, eps=1e-8).run()
    g = ptstokes.Solver(variant, *dims, precision="mixed", lib=gpu_lib, **kw)
    g.setup_inclusion()
    res = g.run()
    assert res["converged"] and res["last"]["err"] <= 1e-8
    for a, b in zip(res["iters"], o.iters):
        assert abs(a - b) <= 100, (res["iters"], o.iters)
    errs = {n: rel(g.get(n), o.f[n]) for n in F3}
    assert max(errs.values()) <= 1e-6, errs
    g.close()


def test_mixed_tracks_fp64_iterates(gpu_lib):
    """Between corrections the FP32 sweeps follow the FP64 iteration: after 3 blocks of
    40 sweeps the FP64 iterate of the mixed path stays close to the plain FP64 one."""
    import ptstokes

    dims = (27, 25, 23)
    p = ptstokes.Solver("3d_ve_perf", *dims, lib=gpu_lib)
    m = ptstokes.Solver("3d_ve_perf", *dims, precision="mixed", lib=gpu_lib)
    for s in (p, m):
        s.setup_inclusion()
        s.assign_tau()
    for _ in range(3):
        p.iterate(40)
        m.iterate(40)
    p.sync()
    m.sync()
    for n in ("Pt", "Vx", "Vz", "txx", "txz"):
        assert rel(m.get(n), p.get(n)) < 1e-5, n
    # the residual is a small difference of large terms: FP32 rounding of δ shows here
    # first (1e-4 relative after 120 sweeps), far below what changes the check's outcome
    cp, cm = p.compute_res(), m.compute_res()
    assert abs(cp["err"] - cm["err"]) <= 1e-3 * cp["err"]
    p.close()
    m.close()


def test_mixed_is_rejected_where_not_implemented(gpu_lib):
    import ptstokes

    with pytest.raises(ptstokes.PtsError):
        ptstokes.Solver("2d_ve", 31, 31, precision="mixed", lib=gpu_lib)


def test_sweep32_kernel_entry(gpu_lib):
    """pts_sweep32_kernel runs one half of an FP32 sweep on a MIXED context's corrections
    (for timing); it refuses other contexts and unknown halves."""
    import ptstokes
    from ptstokes import _abi

    m = ptstokes.Solver("3d_ve_perf", 23, 19, 17, precision="mixed", lib=gpu_lib)
    m.setup_inclusion()
    m.assign_tau()
    m.iterate(4)
    assert gpu_lib.pts_sweep32_kernel(m.ctx, 0) == _abi.PTS_OK
    assert gpu_lib.pts_sweep32_kernel(m.ctx, 1) == _abi.PTS_OK
    assert gpu_lib.pts_sweep32_kernel(m.ctx, 2) == _abi.PTS_E_INVAL
    m.sync()
    m.close()
    p = ptstokes.Solver("3d_ve_perf", 11, 9, 7, lib=gpu_lib)
    assert gpu_lib.pts_sweep32_kernel(p.ctx, 0) == _abi.PTS_E_STATE
    p.close()
