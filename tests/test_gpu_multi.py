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


@pytest.mark.gpu
@pytest.mark.parametrize("nslabs,nz_g", [(2, 26), (3, 32)])
@pytest.mark.parametrize("variant", ["3d_ve", "3d_ve_perf", "3d_v"])
def test_slabs_with_hidden_exchange_equal_one_context(gpu_lib, nslabs, nz_g, variant):
    """@hide_communication b_width (Stokes3D_ve_multixpu.jl:230-239): the end planes of each slab
    are updated first, the halo exchange runs while the inner planes are updated on a second
    stream; the result is still one context of the whole grid, bit for bit."""
    import ptstokes
    from ptstokes.multi import SlabGroup

    nx, ny, iters = 23, 19, 40
    one = ptstokes.Solver(variant, nx, ny, nz_g, lib=gpu_lib, nout=200)
    one.setup_inclusion()
    one.assign_tau()
    one.iterate(iters)
    grp = SlabGroup(variant, nx, ny, nz_g, nslabs, lib=gpu_lib, nout=200, overlap=True)
    grp.setup_inclusion()
    grp.assign_tau()
    for _ in range(iters):
        grp.iteration()
    for k in FIELDS:
        assert np.array_equal(grp.get(k), one.get(k)), k
    err, _ = grp.check()
    assert np.isfinite(err)
    one.close()
    grp.close()


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["3d_ve", "3d_ve_perf"])
def test_plane_ranges_equal_the_whole_update(gpu_lib, variant):
    """compute_V! + bc over disjoint face-plane ranges, launched in any order and on two
    streams, equals the whole update."""
    import ctypes

    import torch

    import ptstokes
    from ptstokes import _abi

    dims = (21, 18, 16)
    a = ptstokes.Solver(variant, *dims, lib=gpu_lib)
    b = ptstokes.Solver(variant, *dims, lib=gpu_lib)
    for s in (a, b):
        s.setup_inclusion()
        s.assign_tau()
        s.iterate(25)
        s.compute_Pt_tau()
        s.sync()  # the side stream's launch below must see compute_Pt_τ!'s results
    a.compute_V_bc()
    side = torch.cuda.Stream()
    nf = dims[2] + 1
    for k0, k1, st in ((9, nf, None), (3, 9, ctypes.c_void_p(side.cuda_stream)), (0, 3, None)):
        assert gpu_lib.pts_compute_V_bc_planes(b.ctx, k0, k1, st) == _abi.PTS_OK
    side.synchronize()
    for s in (a, b):
        s.sync()
    for k in FIELDS[:4]:
        assert np.array_equal(a.get(k), b.get(k)), k
    assert gpu_lib.pts_compute_V_bc_planes(b.ctx, 0, nf + 1, None) == _abi.PTS_E_INVAL
    assert gpu_lib.pts_compute_V_bc_planes(b.ctx, 5, 4, None) == _abi.PTS_E_INVAL
    a.close()
    b.close()
    c = ptstokes.Solver("2d_ve", 15, 13, lib=gpu_lib)
    assert gpu_lib.pts_compute_V_bc_planes(c.ctx, 0, 1, None) == _abi.PTS_E_STATE
    c.close()
