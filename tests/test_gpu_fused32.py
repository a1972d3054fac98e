"""The one-pass FP32 sweep of the mixed path (compute_V! + bc of one sweep and compute_Pt_τ!
of the next in one z-marching kernel; pts_desc.mixed_sweep = 1 + tile) against the default
two-kernel sweeps (mixed_sweep = 0). Both evaluate the same FP32 expressions in the same
order; the compiler contracts some multiply-adds differently in the two kernels, so the
FP32 corrections differ in their last bits and the FP64 iterates by FP32 rounding (relative
to each field's largest value, below 1e-5 after three blocks from the start of a solve,
where the corrections are as large as the fields). A solve to tolerance takes the same
iterations. Grids and chunk sizes cover several tiles in x and y, several z-chunks per
column (chunk boundaries, the z-ghost planes 0 and nz-1 in different chunks), odd and even
numbers of one-pass launches per block."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F = ["Pt", "Vx", "Vy", "Vz", "txx", "tyy", "tzz", "txy", "txz", "tyz"]


def maxrel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pair(gpu_lib, variant, dims, kz, tile):
    import ptstokes

    two = ptstokes.Solver(variant, *dims, precision="mixed", mixed_sweep=0, stencil_kz=kz, lib=gpu_lib)
    one = ptstokes.Solver(variant, *dims, precision="mixed", mixed_sweep=1 + tile, stencil_kz=kz, lib=gpu_lib)
    for s in (two, one):
        s.setup_inclusion()
        s.assign_tau()
    return two, one


@pytest.mark.parametrize("variant", ["3d_ve_perf", "3d_v"])
@pytest.mark.parametrize("dims,m,kz", [((23, 19, 17), 10, 0), ((23, 19, 17), 11, 4), ((70, 37, 21), 9, 5),
                                       ((33, 9, 6), 12, 2)])
@pytest.mark.parametrize("tile", [0, 1, 2])
def test_one_pass_follows_two_kernels(gpu_lib, variant, dims, m, kz, tile):
    two, one = pair(gpu_lib, variant, dims, kz, tile)
    for _ in range(3):
        two.iterate(m)
        one.iterate(m)
    two.sync()
    one.sync()
    d = {n: maxrel(one.get(n), two.get(n)) for n in F}
    assert max(d.values()) <= 1e-5, d
    two.close()
    one.close()


def test_one_pass_solve_iterations(gpu_lib):
    """A solve to 1e-8 (2 physical steps) takes the same iterations either way."""
    import ptstokes

    out = []
    for ms in (0, 1):
        s = ptstokes.Solver("3d_ve_perf", 23, 21, 19, precision="mixed", mixed_sweep=ms, nout=100, nt=2,
                            iter_max=2e5, eps=1e-8, lib=gpu_lib)
        s.setup_inclusion()
        r = s.run()
        assert r["converged"] and r["last"]["err"] <= 1e-8
        out.append((r["iters"], {n: s.get(n) for n in F}))
        s.close()
    assert out[0][0] == out[1][0]
    d = {n: maxrel(out[1][1][n], out[0][1][n]) for n in F}
    assert max(d.values()) <= 1e-6, d


def test_set_mixed_sweep(gpu_lib):
    import ptstokes
    from ptstokes import _abi

    s = ptstokes.Solver("3d_ve_perf", 23, 19, 17, precision="mixed", mixed_sweep=0, lib=gpu_lib)
    s.setup_inclusion()
    s.assign_tau()
    s.iterate(6)
    ntiles = gpu_lib.pts_mixed_sweep_tiles()
    assert ntiles >= 1
    assert gpu_lib.pts_set_mixed_sweep(s.ctx, 1 + ntiles) == _abi.PTS_E_INVAL
    assert gpu_lib.pts_set_mixed_sweep(s.ctx, -1) == _abi.PTS_E_INVAL
    assert gpu_lib.pts_set_mixed_sweep(s.ctx, 1) == _abi.PTS_OK  # allocates the second set here
    s.iterate(6)
    s.sync()
    assert all(np.isfinite(s.get(n)).all() for n in F)
    s.close()
    p = ptstokes.Solver("3d_ve_perf", 11, 9, 7, lib=gpu_lib)
    assert gpu_lib.pts_set_mixed_sweep(p.ctx, 0) == _abi.PTS_E_STATE
    p.close()
