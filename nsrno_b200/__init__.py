"""nsrno_b200: B200-native frequency-domain Helmholtz forward and adjoint solve.

A drop-in for the frequency-domain path of NSRNO (``solve_frequency``,
``solve_system`` and the implicit-gradient ``DenseSurrogate`` path) on a 2-D
variable-density viscoacoustic 5-point Helmholtz operator with a PML.  All
compute runs in hand-written sm_100a CUDA kernels behind the C ABI of
``include/nsrno_b200.h``; this package is the host side.
"""
from . import _lib
from .solver import (BatchResult, Geometry, Medium, Workspace, apply, gmres_batched, grad_accum, plane_wave_rhs,
                     precondition, receiver_response, solve_batched, band_rf, receiver_rf, true_residual)
from .learned import LearnedPreconditioner, LearnedSetup, learned_precondition, warm_start
from .api import (AcquisitionData, HelmholtzSurrogate, HelmholtzSystem, ImplicitChannels, PlaneWaveModel,
                  bin_frequency, implicit_channels, solve_frequency, solve_system)

__all__ = ["BatchResult", "Geometry", "Medium", "Workspace", "apply", "gmres_batched", "grad_accum", "plane_wave_rhs",
           "precondition", "receiver_response", "solve_batched", "AcquisitionData", "HelmholtzSurrogate",
           "HelmholtzSystem", "ImplicitChannels", "PlaneWaveModel", "bin_frequency", "implicit_channels",
           "solve_frequency", "solve_system", "LearnedPreconditioner", "LearnedSetup", "learned_precondition",
           "warm_start", "band_rf", "receiver_rf", "true_residual"]
