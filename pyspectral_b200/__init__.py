"""pyspectral_b200 — B200 (sm_100a) engine for the Lawson IF-RK4 pseudo-spectral
Navier-Stokes step, behind pyspectral's ``SpectralSolver`` interface.

Device work runs in ``libspectral_b200.so`` (C ABI in ``include/spectral_b200.h``): cuFFT
driven from C++, hand-written fused pointwise kernels, one CUDA graph per step.  This package
is the host side: configuration, the solver class, diagnostics and the run driver.
"""

from pyspectral_b200.base import BackendUnavailable, SpectralSolver
from pyspectral_b200.config import Config, fft_split, ffts_per_stage
from pyspectral_b200.registry import REGISTRY, Variant, available, get, make_solver, names

__all__ = ["BackendUnavailable", "SpectralSolver", "Config", "fft_split", "ffts_per_stage",
           "REGISTRY", "Variant", "available", "get", "make_solver", "names"]
