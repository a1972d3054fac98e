"""The z-marching compute_Pt_τ! and compute_V! + bc with TMA-staged planes against the
one-thread-per-point kernels.

FP64: every tile configuration and several z-chunk lengths give the same bits as the direct
kernels after iterations (so the oracle parity of tests/test_gpu_parity.py carries over to
both), on ragged grids whose tiles, z-chunks and halos fall off every edge. The FP32 sweeps
of the mixed path: both kernel forms agree to FP32 rounding. The kernel form can be switched
on a live context.
"""
import numpy as np
import pytest

ITERATED = ("Pt", "Vx", "Vy", "Vz", "txx", "tyy", "tzz", "txy", "txz", "tyz")


def run(gpu_lib, variant, dims, it=12, precision="fp64", **kw):
    """Fields after `it` iterations, assign_τ!, `it` more, and the residual check (its return
    code and result: the smallest grids may go NaN, identically in both kernel forms)."""
    import ctypes

    import ptstokes
    from ptstokes._abi import PtsCheck

    s = ptstokes.Solver(variant, *dims, lib=gpu_lib, nout=it, eps=1e-300, iter_max=10 ** 9, precision=precision,
                        **kw)
    s.setup_inclusion()
    if variant != "3d_v":
        s.assign_tau()
    s.iterate(it)
    if variant != "3d_v":
        s.assign_tau()
    s.iterate(it)
    c = PtsCheck()
    rc = gpu_lib.pts_compute_res(s.ctx, ctypes.byref(c))
    out = {k: s.get(k) for k in ITERATED}
    s.close()
    return out, (rc, bytes(c))


def same_bits(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["3d_ve_perf", "3d_v", "3d_ve"])
@pytest.mark.parametrize("dims", [(37, 29, 23), (33, 7, 40), (4, 3, 5)])
def test_every_tile_is_bit_exact(gpu_lib, variant, dims):
    ref, cref = run(gpu_lib, variant, dims, stencil=1)
    cfgs = [(t, kz, 0) for t in range(gpu_lib.pts_stencil_tiles(0)) for kz in (0, 7, 1)]
    cfgs += [(0, kz, v) for v in range(1, gpu_lib.pts_stencil_vtiles(0)) for kz in (0, 3)]
    for tile, kz, vtile in cfgs:
        got, c = run(gpu_lib, variant, dims, stencil=0, stencil_tile=tile, stencil_kz=kz, stencil_vtile=vtile)
        for k in ITERATED:
            assert same_bits(got[k], ref[k]), (tile, kz, vtile, k)
        assert c == cref


@pytest.mark.gpu
def test_switching_on_a_live_context(gpu_lib):
    import ptstokes

    dims = (41, 35, 29)
    ref, _ = run(gpu_lib, "3d_ve_perf", dims, stencil=1)
    # iter_max = 11: one solve() is exactly one captured block of nout = 12 iterations
    s = ptstokes.Solver("3d_ve_perf", *dims, lib=gpu_lib, nout=12, eps=1e-300, iter_max=11)
    s.setup_inclusion()
    s.assign_tau()
    s.set_stencil(0, gpu_lib.pts_stencil_tiles(0) - 1, 5, gpu_lib.pts_stencil_vtiles(0) - 1)
    s.iterate(5)
    s.set_stencil(1)
    s.iterate(7)
    s.assign_tau()
    s.set_stencil(0, 0, 0)
    assert s.solve()["iters"] == 12  # a captured block after the switch
    for k in ITERATED:
        assert same_bits(s.get(k), ref[k]), k
    with pytest.raises(ptstokes.PtsError):
        s.set_stencil(0, gpu_lib.pts_stencil_tiles(0), 0)
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["3d_ve_perf", "3d_v"])
def test_fp32_sweep_forms_agree(gpu_lib, variant):
    dims = (45, 38, 31)
    ref, _ = run(gpu_lib, variant, dims, it=40, precision="mixed", stencil=1)
    cfgs = [(t, 0) for t in range(gpu_lib.pts_stencil_tiles(1))]
    cfgs += [(0, v) for v in range(1, gpu_lib.pts_stencil_vtiles(1))]
    for tile, vtile in cfgs:
        got, _ = run(gpu_lib, variant, dims, it=40, precision="mixed", stencil=0, stencil_tile=tile,
                     stencil_vtile=vtile)
        for k in ITERATED:
            scale = max(float(np.abs(ref[k]).max()), 1e-300)
            # same FP32 arithmetic up to the compiler's multiply-add contraction
            assert float(np.abs(got[k] - ref[k]).max()) <= 1e-5 * scale, (tile, k)


ITERATED2 = ("Pt", "Vx", "Vy", "txx", "tyy", "txy")


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["2d_ve_perf", "2d_ve", "2d_v"])
@pytest.mark.parametrize("dims", [(47, 39), (33, 70), (65, 9), (3, 3)])
def test_2d_y_marching_tiles_are_bit_exact(gpu_lib, variant, dims):
    """The 2D y-marching compute_Pt_τ! (stencil 0) against the one-thread-per-cell kernel
    (stencil 1): every tile configuration and several rows-per-block chunk lengths, on grids
    whose strips, chunks and halos fall off every edge."""
    import ctypes

    import ptstokes
    from ptstokes._abi import PtsCheck

    def run2(**kw):
        s = ptstokes.Solver(variant, *dims, lib=gpu_lib, nout=9, eps=1e-300, iter_max=10 ** 9, **kw)
        s.setup_inclusion()
        if variant != "2d_v":
            s.assign_tau()
        s.iterate(9)
        if variant != "2d_v":
            s.assign_tau()
        s.iterate(9)
        c = PtsCheck()
        rc = gpu_lib.pts_compute_res(s.ctx, ctypes.byref(c))
        out = {k: s.get(k) for k in ITERATED2}
        s.close()
        return out, (rc, bytes(c))

    ref, cref = run2(stencil=1)
    for tile in range(gpu_lib.pts_stencil_tiles_2d()):
        for ky in (0, 5, 16):
            got, c = run2(stencil=0, stencil_tile=tile, stencil_kz=ky)
            for k in ITERATED2:
                assert same_bits(got[k], ref[k]), (tile, ky, k)
            assert c == cref


@pytest.mark.gpu
@pytest.mark.parametrize("variant,dims", [("3d_ve_perf", (37, 29, 23)), ("2d_ve_perf", (65, 47))])
def test_tune_stencil_picks_a_valid_configuration(gpu_lib, variant, dims):
    import ptstokes

    s = ptstokes.Solver(variant, *dims, lib=gpu_lib, nout=20, eps=1e-300, iter_max=19)
    s.setup_inclusion()
    s.assign_tau()
    e = s.tune_stencil(iters=3, kzs=(8, 0), use_cache=False)
    ntiles = gpu_lib.pts_stencil_tiles(0) if variant.startswith("3d") else gpu_lib.pts_stencil_tiles_2d()
    assert 0 <= e["tile"] < ntiles and e["kz"] in (8, 0)
    assert len(e["ms_per_iteration"]) >= ntiles * 2
    r = s.solve()
    assert r["iters"] == 20 and np.isfinite(r["last"]["err"])
    s.close()
