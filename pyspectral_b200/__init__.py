"""B200-native PySpectral right-hand side and RK4 step.

The hot path -- padded pseudo-spectral RHS of every closure, the fused RK4
stage update and the FP64 diagnostics -- runs in hand-written sm_100a CUDA
(``libpyspectral_b200.so``) behind a C ABI (``include/pyspectral_b200.h``).
The Python modules mirror the reference's operator API:

* :mod:`pyspectral_b200.Classes`      gridclass, FFTclass, variables, utilitiesClass
* :mod:`pyspectral_b200.RHSfunctions` computeRHS_NOSGS/SMAG/tmodel/staumodel/Dtaumodel, advanceQ_RK4
* :mod:`pyspectral_b200.mpi`          MHD of the MPI solver (computeRHS_MHD, advanceQ_RK4, diagnostics)
* :mod:`pyspectral_b200.initial_conditions` TGV and isotropic initial fields
"""
from . import _capi  # noqa: F401

__all__ = ["_capi"]
