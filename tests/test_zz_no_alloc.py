"""pts_check_noalloc: the convergence check for callers that cannot allocate.

A caller whose device memory all belongs to another allocator (a Julia program using
CUDA.jl's pool, a PyTorch program using the caching allocator) or that forbids cudaMalloc
after start-up hands its own arrays to pts_check_noalloc; the library keeps the block
partials of the reduction in a fixed array of its own and allocates nothing. Here the
caller's arrays are torch tensors filled from a solver context, and the result must equal
the context's own check (pts_compute_res) to the 1e-12 relative tolerance the other
check tests use, on two calls in a row (the second call reuses the shared array).
"""
import ctypes

import numpy as np
import pytest

CHECK_KEYS = ("err", "norm_Rx", "norm_Ry", "norm_Rz", "norm_divV", "Vmin", "Vmax", "Pmin", "Pmax")


@pytest.mark.gpu
@pytest.mark.parametrize("variant,dims", [("3d_ve_perf", (41, 37, 33)), ("3d_v", (35, 33, 31)),
                                          ("2d_ve_perf", (63, 47)),
                                          # 2 x 32 tiles per plane: 64 z-blocks for 200 planes, so each
                                          # block reduces several strided planes
                                          ("3d_v", (63, 255, 200))])
def test_noalloc_check_matches_the_context_check(gpu_lib, variant, dims):
    import torch

    import ptstokes
    from ptstokes import _abi

    s = ptstokes.Solver(variant, *dims, lib=gpu_lib)
    s.setup_inclusion()
    s.assign_tau()
    s.iterate(30)
    ref = s.compute_res()
    expected = np.array([ref[k] for k in CHECK_KEYS])

    # the caller's own device arrays (dense, the reference's extents)
    owned = {}
    ptrs = (ctypes.c_void_p * 10)()
    for q, name in enumerate(_abi.FIELDS[:10]):
        if s.ndim == 2 and name in ("Vz", "tzz", "txz", "tyz"):
            continue
        n = int(np.prod(s.shape(name)))
        t = torch.empty(n, dtype=torch.float64, device="cuda")
        s.get_device(name, t.data_ptr(), n)
        owned[name] = t
        ptrs[q] = t.data_ptr()
    out = torch.empty(len(CHECK_KEYS), dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = gpu_lib.pts_check_noalloc(ctypes.byref(s.desc), ptrs, ctypes.c_void_p(out.data_ptr()), None)
        assert rc == _abi.PTS_OK, gpu_lib.pts_last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, expected, rtol=1e-12, atol=0)
    s.close()


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch():
    """The size check comes before any CUDA call, so it runs without a GPU."""
    import ptstokes
    from ptstokes import _abi

    lib = ptstokes.load()
    d = _abi.PtsDesc()
    d.variant, d.nx, d.ny, d.nz = _abi.VARIANTS["3d_ve_perf"], 2047, 2047, 8
    d.lx = d.ly = d.lz = 10.0
    ptrs = (ctypes.c_void_p * 10)(*([16] * 10))  # never dereferenced: rejected first
    rc = lib.pts_check_noalloc(ctypes.byref(d), ptrs, ctypes.c_void_p(16), None)
    assert rc == _abi.PTS_E_INVAL
    assert b"at most 4096" in lib.pts_last_error(None)
    d.variant = _abi.VARIANTS["3d_ve"]
    d.nx = d.ny = 63
    assert lib.pts_check_noalloc(ctypes.byref(d), ptrs, ctypes.c_void_p(16), None) == _abi.PTS_E_INVAL
    # domain extents that would make the 1/dx factors infinite or NaN
    d.variant = _abi.VARIANTS["3d_ve_perf"]
    for lx, lz in ((0.0, 10.0), (-1.0, 10.0), (float("nan"), 10.0), (10.0, 0.0)):
        d.lx, d.lz = lx, lz
        assert lib.pts_check_noalloc(ctypes.byref(d), ptrs, ctypes.c_void_p(16), None) == _abi.PTS_E_INVAL
        assert b"extents" in lib.pts_last_error(None)
