"""CPU oracle for the pseudo-transient Stokes path -- TEST INFRASTRUCTURE ONLY.

This package restates the reference (PTsolvers/PseudoTransientStokes.jl) on the CPU:
``ptstokes_oracle.cpp`` holds the stencil kernels (C++17/OpenMP, FP64, no FMA
contraction) and ``scripts.py`` holds the drivers that mirror each reference
script's ``Stokes2D_()`` / ``Stokes3D_()`` function.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may
import it, and only as the checker; the product package never does.
"""
from .binding import lib, build, Arr, arr  # noqa: F401
from . import scripts  # noqa: F401
