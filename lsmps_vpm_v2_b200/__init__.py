"""B200-native FMM velocity step of the LSMPS vortex particle method.

The compute path is libvpm_fmm.so (hand-written sm_100a CUDA kernels behind
the C ABI in include/vpm_fmm.h); this package binds it and mirrors the
reference's operator interface for the path.
"""
from ._lib import (BINOM_EXACT, BINOM_REFERENCE, PREC_FP64, PREC_MIXED, Params, Stats, VpmError,
                   default_params, lib, treecell3d_params)
from .fmm import Context, Particle, TreeCell, VelocityCalc, default_context, fmm2D, fmm3D
from .state import read_particle_state, write_particle_state

__all__ = [
    "BINOM_EXACT", "BINOM_REFERENCE", "PREC_FP64", "PREC_MIXED", "Params", "Stats", "VpmError", "fmm3D",
    "default_params", "lib", "Context", "Particle", "TreeCell", "VelocityCalc", "default_context", "fmm2D",
    "read_particle_state", "write_particle_state", "treecell3d_params",
]
