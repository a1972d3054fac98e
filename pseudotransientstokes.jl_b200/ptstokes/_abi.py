"""ctypes binding of libptstokes.so (the C ABI declared in include/ptstokes.h).

The shared library is the product: there is no Python or CPU fallback. If it is missing
or cannot be loaded, ``load()`` raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "lib", "libptstokes.so"))

PTS_OK = 0
PTS_E_INVAL = -1
PTS_E_CUDA = -2
PTS_E_NOMEM = -3
PTS_E_NAN = -4
PTS_E_STATE = -5

VARIANTS = {
    "2d_v": 0,        # scripts/Stokes2D.jl
    "2d_ve": 1,       # scripts/Stokes2D_ve.jl
    "2d_ve_perf": 2,  # scripts/Stokes2D_ve_perf.jl
    "3d_ve": 3,       # scripts/stokes_3D/Stokes3D_ve_multixpu.jl (one rank)
    "3d_ve_perf": 4,  # scripts/stokes_3D/Stokes3D_ve_perf.jl
    "3d_v": 5,        # 3D viscous (no reference script)
    "2d_v_damp": 6,   # scripts/previous_damp/Stokes2D0.jl
    "2d_ve_damp": 7,  # scripts/previous_damp/Stokes2D_ve0.jl
    "3d_v_damp": 8,   # scripts/stokes_3D/previous_damp/Stokes3D0_multixpu.jl (one rank)
}
PRECISIONS = {"fp64": 0, "mixed": 1}

FIELDS = [
    "Pt", "Vx", "Vy", "Vz",
    "txx", "tyy", "tzz", "txy", "txz", "tyz",
    "txx_o", "tyy_o", "tzz_o", "txy_o", "txz_o", "tyz_o",
    "Mus", "Must", "Gdt", "dtRho", "divV",
    "Rx", "Ry", "Rz", "dVx", "dVy", "dVz",
    "rhog",
    "Fx", "Fy", "Fz",
    "grad",
    "dtVx", "dtVy", "dtVz", "dtPt",
]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}


class PtsDesc(ctypes.Structure):
    _fields_ = [
        ("variant", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("nout", ctypes.c_int32),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("G", ctypes.c_double), ("dt", ctypes.c_double),
        ("r", ctypes.c_double), ("Re", ctypes.c_double), ("CFL", ctypes.c_double),
        ("max_l", ctypes.c_double), ("eps", ctypes.c_double), ("iter_max", ctypes.c_double),
        ("mixed_inner", ctypes.c_int32), ("single_pass", ctypes.c_int32), ("adjoint", ctypes.c_int32),
        ("stencil", ctypes.c_int32), ("stencil_tile", ctypes.c_int32), ("stencil_kz", ctypes.c_int32),
        ("stencil_vtile", ctypes.c_int32), ("mixed_sweep", ctypes.c_int32),
    ]


class PtsCheck(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("err", "norm_Rx", "norm_Ry", "norm_Rz", "norm_divV", "Vmin", "Vmax", "Pmin", "Pmax")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class PtsSolveInfo(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int64), ("converged", ctypes.c_int32), ("nchecks", ctypes.c_int32),
                ("last", PtsCheck)]


class PtsInclusion(ctypes.Structure):
    _fields_ = [("x", ctypes.c_double), ("y", ctypes.c_double), ("z", ctypes.c_double), ("r2", ctypes.c_double),
                ("mus", ctypes.c_double)]


class PtsBatchInstance(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("lx", ctypes.c_double), ("ly", ctypes.c_double),
                ("musi", ctypes.c_double), ("radius2", ctypes.c_double), ("rhogi", ctypes.c_double),
                ("ebg", ctypes.c_double)]


class PtsBatchVEInstance(ctypes.Structure):
    _fields_ = [("ny", ctypes.c_int32), ("nsub", ctypes.c_int32), ("nt", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("fact", ctypes.c_double), ("ly", ctypes.c_double),
                ("musi", ctypes.c_double)]


class PtsBatchDesc(ctypes.Structure):
    _fields_ = [("nout", ctypes.c_int32), ("tile", ctypes.c_int32), ("eps", ctypes.c_double),
                ("iter_max", ctypes.c_double), ("r", ctypes.c_double), ("Re", ctypes.c_double),
                ("CFL", ctypes.c_double), ("reserved", ctypes.c_int32 * 4)]


class PtsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ptstokes error {code}: {msg}")
        self.code = code


_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double
_DP = ctypes.c_void_p  # double* (host or device), passed as an address

SIGNATURES = {
    "pts_abi_version": ([], ctypes.c_int),
    "pts_stencil_tiles": ([_I32], ctypes.c_int),
    "pts_stencil_vtiles": ([_I32], ctypes.c_int),
    "pts_set_stencil": ([_P, _I32, _I32, _I32, _I32], ctypes.c_int),
    "pts_stencil_tile_info": ([_I32, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_I32)], ctypes.c_int),
    "pts_last_error": ([_P], ctypes.c_char_p),
    "pts_create": ([ctypes.POINTER(PtsDesc), ctypes.POINTER(_P)], ctypes.c_int),
    "pts_destroy": ([_P], ctypes.c_int),
    "pts_sync": ([_P], ctypes.c_int),
    "pts_stream": ([_P, ctypes.POINTER(_P)], ctypes.c_int),
    "pts_field_shape": ([_P, _I32, ctypes.POINTER(_I64)], ctypes.c_int),
    "pts_set_field": ([_P, _I32, _DP, _I64], ctypes.c_int),
    "pts_get_field": ([_P, _I32, _DP, _I64], ctypes.c_int),
    "pts_set_field_device": ([_P, _I32, _DP, _I64], ctypes.c_int),
    "pts_get_field_device": ([_P, _I32, _DP, _I64], ctypes.c_int),
    "pts_init_inclusion": ([_P, _D, _D, _D, _D], ctypes.c_int),
    "pts_init_inclusions": ([_P, ctypes.POINTER(PtsInclusion), _I32, _D, _D], ctypes.c_int),
    "pts_smooth": ([_P, _I32, _D], ctypes.c_int),
    # z-slab decomposition (ptstokes.multi)
    "pts_set_decomposition": ([_P, _I32, _I32], ctypes.c_int),
    "pts_get_plane_device": ([_P, _I32, _I32, _DP, _I64], ctypes.c_int),
    "pts_set_plane_device": ([_P, _I32, _I32, _DP, _I64], ctypes.c_int),
    "pts_check_partials": ([_P, ctypes.POINTER(_D)], ctypes.c_int),
    "pts_set_norm_scales": ([_P, _D, _D, _D, _D], ctypes.c_int),
    "pts_set_mixed_sweep": ([_P, ctypes.c_int32], ctypes.c_int),
    "pts_mixed_sweep_tiles": ([], ctypes.c_int),
    "pts_stencil_tiles_2d": ([], ctypes.c_int),
    "pts_compute_maxloc": ([_P], ctypes.c_int),
    "pts_compute_iter_params": ([_P], ctypes.c_int),
    "pts_set_damping": ([_P] + [ctypes.c_double] * 4, ctypes.c_int),
    "pts_assign_tau": ([_P], ctypes.c_int),
    "pts_compute_P": ([_P], ctypes.c_int),
    "pts_compute_tau": ([_P], ctypes.c_int),
    "pts_compute_dV": ([_P], ctypes.c_int),
    "pts_compute_V": ([_P], ctypes.c_int),
    "pts_apply_bc": ([_P], ctypes.c_int),
    "pts_compute_Pt_tau": ([_P], ctypes.c_int),
    "pts_compute_V_bc": ([_P], ctypes.c_int),
    "pts_sweep32_kernel": ([_P, ctypes.c_int32], ctypes.c_int),
    "pts_set_kernel_timing": ([_P, ctypes.c_int32], ctypes.c_int),
    "pts_kernel_times": ([_P, ctypes.POINTER(ctypes.c_float), ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)],
                         ctypes.c_int),
    "pts_compute_res": ([_P, ctypes.POINTER(PtsCheck)], ctypes.c_int),
    "pts_iterate": ([_P, _I64], ctypes.c_int),
    "pts_solve": ([_P, ctypes.POINTER(PtsSolveInfo)], ctypes.c_int),
    "pts_run": ([_P, _I32, ctypes.POINTER(_I64), ctypes.POINTER(PtsSolveInfo)], ctypes.c_int),
    # adjoint of the 3D viscous solve
    "pts_apply_operator": ([_P, ctypes.POINTER(PtsCheck)], ctypes.c_int),
    "pts_gradient_logmu": ([_P, _P], ctypes.c_int),
    "pts_gradient_logmu_add": ([_P, _P], ctypes.c_int),
    # residual check on caller-owned device arrays; allocates nothing
    "pts_compute_V_bc_planes": ([_P, _I32, _I32, _P], ctypes.c_int),
    "pts_check_noalloc": ([ctypes.POINTER(PtsDesc), ctypes.POINTER(_P), _P, _P], ctypes.c_int),
    # batched 2D sweep
    "pts_batch_create": ([ctypes.POINTER(PtsBatchDesc), ctypes.POINTER(PtsBatchInstance), _I32, ctypes.POINTER(_P)],
                         ctypes.c_int),
    "pts_batch_destroy": ([_P], ctypes.c_int),
    "pts_batch_last_error": ([_P], ctypes.c_char_p),
    "pts_batch_setup": ([_P], ctypes.c_int),
    "pts_batch_set_tile": ([_P, _I32], ctypes.c_int),
    "pts_batch_solve": ([_P, _I64, ctypes.POINTER(_I64), ctypes.POINTER(_D), ctypes.POINTER(_I32),
                         ctypes.POINTER(_I32)], ctypes.c_int),
    "pts_batch_get_field": ([_P, _I32, _I32, _DP, _I64], ctypes.c_int),
    "pts_batch_stream": ([_P, ctypes.POINTER(_P)], ctypes.c_int),
    # batched 2D visco-elastic aspect-ratio sweep
    "pts_batch_create_ve": ([ctypes.POINTER(PtsBatchDesc), ctypes.POINTER(PtsBatchVEInstance), _I32,
                             ctypes.POINTER(_P)], ctypes.c_int),
    "pts_batch_steps": ([_P, _I32, ctypes.POINTER(_I64), _I32, ctypes.POINTER(_I32)], ctypes.c_int),
}

_lib = None


def load(path=None):
    """Load libptstokes.so and declare the C signatures. Raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("PTSTOKES_LIB") or LIB_PATH
    if not os.path.exists(p):
        raise OSError(f"libptstokes.so not found at {p}; build it with "
                      f"`python pseudotransientstokes.jl_b200/build.py`")
    lib = ctypes.CDLL(p)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _lib = lib
    return lib


def check(lib, ctx, rc):
    if rc != PTS_OK:
        msg = lib.pts_last_error(ctx)
        raise PtsError(rc, msg.decode() if msg else "")
    return rc
