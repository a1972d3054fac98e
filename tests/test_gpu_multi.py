"""The z-slab decomposition on the GPU (ptstokes.multi.SlabGroup): two and three slab
contexts of Stokes3D_ve_multixpu.jl's problem, their halo planes exchanged by device copies
after every PT iteration (update_halo!) and during set-up (Mus, Musτ), equal one context
of the whole grid bit for bit; the check reduced over the slabs counts the overlap planes
twice, as the reference's norm_g does. (The exchange between processes, over NCCL, is the
same plane traffic through torch.distributed; its host logic is tested on gloo ranks in
tests/test_multi_cpu.py.)"""
import numpy as np
import pytest

FIELDS = ("Pt", "Vx", "Vy", "Vz", "txx", "tyy", "tzz", "txy", "txz", "tyz", "Mus", "Must")


@pytest.mark.gpu
@pytest.mark.parametrize("nslabs,nz_g", [(2, 26), (3, 32)])
@pytest.mark.parametrize("variant", ["3d_ve", "3d_ve_perf"])
def test_slabs_equal_one_context(gpu_lib, nslabs, nz_g, variant):
    import ptstokes
    from ptstokes.multi import SlabGroup

    nx, ny, iters = 23, 19, 40
    one = ptstokes.Solver(variant, nx, ny, nz_g, lib=gpu_lib, nout=200)
    one.setup_inclusion()
    one.assign_tau()
    one.iterate(iters)
    grp = SlabGroup(variant, nx, ny, nz_g, nslabs, lib=gpu_lib, nout=200)
    grp.setup_inclusion()
    grp.assign_tau()
    for _ in range(iters):
        grp.iteration()
    for k in FIELDS:
        got, want = grp.get(k), one.get(k)
        assert got.shape == want.shape, k
        assert np.array_equal(got, want), k
    err, norms = grp.check()
    ref = one.compute_res()
    assert np.isfinite(err) and abs(err - ref["err"]) <= 0.2 * ref["err"]
    one.close()
    grp.close()


@pytest.mark.gpu
def test_decomposition_rejects_bad_slabs(gpu_lib):
    import ptstokes
    from ptstokes import _abi

    s = ptstokes.Solver("3d_ve", 11, 9, 8, lib=gpu_lib)
    assert gpu_lib.pts_set_decomposition(s.ctx, 5, 12) == _abi.PTS_E_INVAL  # slab past the end
    assert gpu_lib.pts_set_decomposition(s.ctx, -1, 20) == _abi.PTS_E_INVAL
    assert gpu_lib.pts_set_decomposition(s.ctx, 4, 12) == _abi.PTS_OK
    s.close()
    t = ptstokes.Solver("2d_v", 11, 9, lib=gpu_lib)
    assert gpu_lib.pts_set_decomposition(t.ctx, 0, 9) == _abi.PTS_E_STATE
    t.close()
