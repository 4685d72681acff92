"""shtns_b200: spherical harmonic transforms on NVIDIA B200 (sm_100a) behind the
SHTns 3.5.2 C API.

The compute path is the C-ABI library libshtns_b200.so (hand-written CUDA);
this package only binds it.  Importing the transform classes loads the library
and fails loudly if it was not built.
"""
from .capi import (sht_orthonormal, sht_fourpi, sht_schmidt, SHT_NO_CS_PHASE, SHT_REAL_NORM,  # noqa: F401
                   sht_gauss, sht_auto, sht_reg_fast, sht_reg_dct, sht_quick_init, sht_reg_poles, sht_gauss_fly,
                   SHT_NATIVE_LAYOUT, SHT_THETA_CONTIGUOUS, SHT_PHI_CONTIGUOUS, SHT_SOUTH_POLE_FIRST,
                   SHT_SCALAR_ONLY, SHT_LOAD_SAVE_CFG, SHT_ALLOW_GPU, SHT_ALLOW_PADDING, SHTError)

from .transforms import sht, rotation  # noqa: F401  (the CUDA library loads when a plan is created)

__version__ = "0.1.0"


# Module-level functions of the reference's Python module, which exposes the
# free functions of shtns.h (shtns_numpy.i:131-135 renames three of them).

def nlm_calc(lmax, mmax, mres):
    """Number of real-field spherical harmonic coefficients (shtns.h:133)."""
    from . import capi
    return int(capi.load().nlm_calc(int(lmax), int(mmax), int(mres)))


def nlm_cplx_calc(lmax, mmax, mres):
    """Number of complex-field coefficients, orders -mmax..mmax (shtns.h:136)."""
    from . import capi
    return int(capi.load().nlm_cplx_calc(int(lmax), int(mmax), int(mres)))


def set_verbosity(level):
    """shtns_verbose (shtns.h:138): 0 silent, higher values print plan details."""
    from . import capi
    capi.load().shtns_verbose(int(level))


def print_version():
    """shtns_print_version (shtns.h:139)."""
    from . import capi
    capi.load().shtns_print_version()


def build_info():
    """shtns_get_build_info (shtns.h:140): the library's build description."""
    from . import capi
    info = capi.load().shtns_get_build_info()
    return info.decode() if isinstance(info, bytes) else info


def shtns_use_threads(num_threads):
    """shtns_use_threads (shtns.h:159); this library computes on the GPU."""
    from . import capi
    return int(capi.load().shtns_use_threads(int(num_threads)))


def shtns_use_gpu(device_id):
    """shtns_use_gpu (shtns.h:161): selects the CUDA device for later plans."""
    from . import capi
    return int(capi.load().shtns_use_gpu(int(device_id)))
