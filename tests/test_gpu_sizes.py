"""Edge sizes on the GPU, through the C ABI.

* The smallest grids the stencils allow (3 cells along an axis, where each stress and
  velocity interior is a single plane) and ragged shapes whose x-faces fill the padded row
  exactly (nx + 1 = 16 or 32) or spill one face into the next 16-element group (nx = 16),
  for every variant: every field bit for bit against
  the oracle after a few PT iterations (NaN where the oracle has NaN).
* A full-size case: 3D VE (Stokes3D_ve_perf.jl kernels) at 255^3, three iterations, bit for
  bit against the oracle.
* The benchmark's size, 511^3: the set-up and three PT iterations of the Stokes3D_ve_perf.jl
  problem bit for bit against the oracle (the z-marching kernels, the default), and the
  single-pass kernels against the two-kernel path.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VARIANTS = ["2d_v", "2d_ve", "2d_ve_perf", "2d_v_damp", "2d_ve_damp", "3d_ve", "3d_ve_perf", "3d_v", "3d_v_damp"]
SMALL2 = [(3, 3), (3, 5), (15, 3), (16, 4), (31, 6)]
SMALL3 = [(3, 3, 3), (3, 4, 5), (15, 3, 4), (16, 5, 3)]
F2 = ["Pt", "Vx", "Vy", "txx", "tyy", "txy"]
F3 = F2 + ["Vz", "tzz", "txz", "tyz"]


def _pair(gpu_lib, variant, dims):
    import ptstokes
    from oracle import scripts as S
    o = S.make(variant, *dims)
    g = ptstokes.Solver(variant, *dims, lib=gpu_lib)
    g.setup_inclusion()
    return o, g


def _equal(o, g, names):
    bad = []
    for n in names:
        a, b = g.get(n), o.f[n]
        assert a.shape == b.shape, (n, a.shape, b.shape)
        if not np.array_equal(a, b, equal_nan=True):
            bad.append((n, float(np.nanmax(np.abs(a - b)))))
    assert not bad, bad


def _cases():
    for v in VARIANTS:
        for d in (SMALL3 if v.startswith("3d") else SMALL2):
            yield v, d


@pytest.mark.parametrize("variant,dims", list(_cases()))
def test_small_and_ragged_grids_bit_exact(gpu_lib, variant, dims):
    o, g = _pair(gpu_lib, variant, dims)
    if o.elastic:
        o.assign_tau()
        g.assign_tau()
    with np.errstate(all="ignore"):
        for _ in range(7):
            o.iteration()
    g.iterate(7)
    g.sync()
    _equal(o, g, ["Mus", "Must"] + (F3 if variant.startswith("3d") else F2))
    g.close()


def test_full_size_255_bit_exact(gpu_lib):
    o, g = _pair(gpu_lib, "3d_ve_perf", (255, 255, 255))
    o.assign_tau()
    g.assign_tau()
    for _ in range(3):
        o.iteration()
    g.iterate(3)
    g.sync()
    _equal(o, g, F3)
    g.close()


def test_full_size_511_bit_exact(gpu_lib):
    o, g = _pair(gpu_lib, "3d_ve_perf", (511, 511, 511))
    o.assign_tau()
    g.assign_tau()
    for _ in range(3):
        o.iteration()
    g.iterate(3)
    g.sync()
    _equal(o, g, ["Mus", "Must"] + F3)
    g.close()


def test_511_single_pass_equals_two_kernel_path(gpu_lib):
    import ptstokes
    n = 511
    a = ptstokes.Solver("3d_ve_perf", n, n, n, lib=gpu_lib)
    a.setup_inclusion()
    a.assign_tau()
    a.iterate(5)
    a.sync()
    ref = {k: a.get(k) for k in F3}
    a.close()
    for mode in (1, 2):
        b = ptstokes.Solver("3d_ve_perf", n, n, n, lib=gpu_lib, single_pass=mode)
        b.setup_inclusion()
        b.assign_tau()
        b.iterate(5)
        b.sync()
        for k in F3:
            assert np.array_equal(b.get(k), ref[k]), (mode, k)
        b.close()
