"""shtns_b200: spherical harmonic transforms on NVIDIA B200 (sm_100a) behind the
SHTns 3.5.2 C API.

The compute path is the C-ABI library libshtns_b200.so (hand-written CUDA);
this package only binds it.  Importing the transform classes loads the library
and fails loudly if it was not built.
"""
from .capi import (sht_orthonormal, sht_fourpi, sht_schmidt, SHT_NO_CS_PHASE, SHT_REAL_NORM,  # noqa: F401
                   sht_gauss, sht_auto, sht_quick_init, sht_gauss_fly,
                   SHT_NATIVE_LAYOUT, SHT_THETA_CONTIGUOUS, SHT_PHI_CONTIGUOUS, SHT_SOUTH_POLE_FIRST,
                   SHT_SCALAR_ONLY, SHT_ALLOW_GPU, SHTError)

from .transforms import sht, rotation  # noqa: F401  (the CUDA library loads when a plan is created)

__version__ = "0.1.0"
