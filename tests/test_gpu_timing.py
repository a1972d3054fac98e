"""Per-kernel timing (pts_set_kernel_timing / pts_kernel_times): a CUDA event after each
kernel of a block of PT iterations, inside the check block's graph; the fields are the same
bits with and without it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F = ["Pt", "Vx", "Vy", "Vz", "txx", "tyy", "tzz", "txy", "txz", "tyz"]


@pytest.mark.parametrize("variant,dims", [("3d_ve_perf", (23, 19, 17)), ("2d_ve_perf", (47, 39))])
def test_kernel_times_of_graph_blocks(gpu_lib, variant, dims):
    import ptstokes

    out = []
    for timing in (False, True):
        s = ptstokes.Solver(variant, *dims, nout=10, eps=1e-300, iter_max=9, lib=gpu_lib)
        s.set_kernel_timing(timing)
        s.setup_inclusion()
        s.assign_tau()
        for _ in range(3):
            s.solve()  # graph blocks of 10 iterations + check
        t = s.kernel_times()
        if timing:
            assert len(t) == 2 * 10 + 1  # compute_Pt_τ!, compute_V! + bc per iteration, the check
            assert all(x > 0 for x in t)
        else:
            assert t == []
        out.append({n: s.get(n) for n in F if n in ("Pt", "Vx", "Vy", "txx", "txy") or variant.startswith("3d")})
        s.close()
    for n in out[0]:
        assert np.array_equal(out[0][n], out[1][n]), n


def test_kernel_times_mixed_and_direct(gpu_lib):
    """Mixed blocks record the two FP32 half-sweeps per sweep, the fold and the check; a block
    enqueued directly (pts_iterate) records its kernels too."""
    import ptstokes

    m = ptstokes.Solver("3d_ve_perf", 23, 19, 17, precision="mixed", nout=10, eps=1e-300, iter_max=9, lib=gpu_lib)
    m.set_kernel_timing(True)
    m.setup_inclusion()
    m.assign_tau()
    m.solve()
    assert len(m.kernel_times()) == 2 * 10 + 2
    m.close()
    p = ptstokes.Solver("3d_ve_perf", 23, 19, 17, lib=gpu_lib)
    p.set_kernel_timing(True)
    p.setup_inclusion()
    p.assign_tau()
    p.iterate(7)
    assert len(p.kernel_times()) == 2 * 7
    p.close()
