"""ptstokes -- Python host of libptstokes.so, the B200 pseudo-transient Stokes solver.

A drop-in for the hot path of PTsolvers/PseudoTransientStokes.jl: ``Solver`` exposes
the reference's kernel roles on device-resident fields; ``scripts`` mirrors each
reference script's solver function; ``batch`` runs parameter sweeps of many uneven
instances in one persistent launch. All compute runs in the CUDA library.
"""
from ._abi import PtsError, load, FIELDS, VARIANTS  # noqa: F401
from .solver import Solver, VARIANT_DEFAULTS, linrange  # noqa: F401
from . import scripts  # noqa: F401
from . import batch  # noqa: F401
