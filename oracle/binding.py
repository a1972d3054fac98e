"""ctypes binding of the oracle's C kernels (test infrastructure only)."""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "ptstokes_oracle.cpp")
_SO = os.path.join(_HERE, "_build", "libptsoracle.so")

# -ffp-contract=off: no fused multiply-add, matching Julia's evaluation of the reference.
CXXFLAGS = ["-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared"]


def build(force=False):
    """Compile the oracle into oracle/_build/libptsoracle.so (g++ / OpenMP)."""
    os.makedirs(os.path.dirname(_SO), exist_ok=True)
    if not force and os.path.exists(_SO) and os.path.getmtime(_SO) >= os.path.getmtime(_SRC):
        return _SO
    subprocess.check_call(["g++", *CXXFLAGS, _SRC, "-o", _SO])
    return _SO


class Arr(ctypes.Structure):
    _fields_ = [("p", ctypes.c_void_p), ("n1", ctypes.c_int64), ("n2", ctypes.c_int64), ("n3", ctypes.c_int64)]


def arr(a):
    """View a Fortran-ordered float64 numpy array as the oracle's ``oarr``."""
    if a is None:
        return Arr(None, 0, 0, 0)
    assert a.dtype == np.float64 and a.flags.f_contiguous, "oracle arrays are Float64 column-major"
    s = list(a.shape) + [1] * (3 - a.ndim)
    return Arr(a.ctypes.data, s[0], s[1], s[2])


_lib = None

_D = ctypes.c_double
_I = ctypes.c_int
_L = ctypes.c_int64

_SIGS = {
    "ora_copy": [Arr, Arr],
    "ora_iter_params_v": [Arr, Arr, Arr, _D, _D, _D, _D],
    "ora_iter_params_ve": [Arr, Arr, Arr, _D, _D, _D, _D, _D, _D],
    "ora2_smooth": [Arr, Arr, _D],
    "ora2_maxloc": [Arr, Arr],
    "ora2_bc_x": [Arr],
    "ora2_bc_y": [Arr],
    "ora2_compute_P": [Arr, Arr, Arr, Arr, Arr, _D, _D, _D],
    "ora2v_compute_tau": [Arr, Arr, Arr, Arr, Arr, Arr, Arr, _D, _D],
    "ora2v_compute_dV": [Arr] * 9 + [_D, _D],
    "ora2_compute_V": [Arr] * 4,
    "ora2ve_compute_tau": [Arr] * 10 + [_D, _D, _D, _D],
    "ora2ve_compute_dV": [Arr] * 7 + [_D, _D],
    "ora2ve_compute_Res": [Arr] * 6 + [_D, _D],
    "ora2p_compute_Pt_tau": [Arr] * 11 + [_D] * 5,
    "ora2p_compute_V": [Arr] * 7 + [_D, _D, _L, _L, _L, _L],
    "ora2p_compute_Res": [Arr] * 9 + [_D, _D],
    "ora2_create_inclusions": [Arr, Arr, ctypes.c_void_p, ctypes.c_void_p, _L] + [_D] * 9,
    "ora_create_inclusions_list": [Arr] + [ctypes.c_void_p] * 5 + [_L] + [_D] * 7 + [ctypes.c_int],
    "ora2s_compute_tau": [Arr] * 7 + [_D, _D],
    "ora2s_compute_dV": [Arr] * 10 + [_D, _D],
    "ora3_smooth": [Arr, Arr, _D],
    "ora3_maxloc": [Arr, Arr],
    "ora3_bc_x": [Arr],
    "ora3_bc_y": [Arr],
    "ora3_bc_z": [Arr],
    "ora3m_compute_P": [Arr] * 6 + [_D] * 4,
    "ora3m_compute_tau": [Arr] * 17 + [_D] * 5 + [_I],
    "ora3m_compute_dV": [Arr] * 11 + [_D] * 3 + [_I],
    "ora3_compute_V": [Arr] * 6,
    "ora3p_compute_Pt_tau": [Arr] * 18 + [_D] * 6 + [_I],
    "ora3p_compute_V": [Arr] * 11 + [_D] * 3,
    "ora3p_compute_V_src": [Arr] * 14 + [_D] * 3,
    "ora3v_tau_exact": [Arr] * 10 + [_D] * 3,
    "ora3v_grad_logmu": [Arr] * 8 + [_D] * 3,
    "ora3v_res_adj": [Arr] * 10 + [_D] * 3,
    "ora3v_update_V": [Arr] * 10,
    "ora3ve_grad_logmu": [Arr] * 14 + [ctypes.c_int],
    "ora2d_timesteps": [Arr] * 4 + [_D] * 5,
    "ora2d_compute_P": [Arr] * 5 + [_D] * 2,
    "ora2d_compute_tau": [Arr] * 10 + [_D] * 5 + [ctypes.c_int],
    "ora2d_compute_dV": [Arr] * 8 + [_D] * 4,
    "ora2d_compute_V": [Arr] * 6,
    "ora3d_timesteps": [Arr] * 5 + [_D] * 5,
    "ora3d_compute_P": [Arr] * 6 + [_D] * 3,
    "ora3d_compute_tau": [Arr] * 11 + [_D] * 4,
    "ora3d_compute_dV": [Arr] * 13 + [_D] * 6,
    "ora3d_compute_V": [Arr] * 9,
    "ora3p_compute_Res": [Arr] * 14 + [_D] * 3,
    "ora_stats": [Arr, ctypes.POINTER(_D), ctypes.POINTER(_D), ctypes.POINTER(_D)],
    "ora_num_threads": [],
}


def lib():
    """Load (building first if needed) the oracle shared library."""
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        for name, argtypes in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = argtypes
            f.restype = ctypes.c_int if name == "ora_num_threads" else None
        _lib = L
    return _lib


def stats(a):
    """(sum of squares, min, max) of a whole array."""
    s, lo, hi = _D(), _D(), _D()
    lib().ora_stats(arr(a), ctypes.byref(s), ctypes.byref(lo), ctypes.byref(hi))
    return s.value, lo.value, hi.value
