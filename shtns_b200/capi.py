"""ctypes declarations of the shtns_b200 C ABI (include/shtns.h,
include/shtns_cuda.h, include/shtns_b200.h).

The shared library is built in-tree (shtns_b200/libshtns_b200.so) by
shtns_b200/build.py.  Loading fails with ImportError when it is missing: there
is no CPU fallback.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libshtns_b200.so")

# enums and flags (shtns.h:48-75)
sht_orthonormal, sht_fourpi, sht_schmidt = 0, 1, 2
SHT_NO_CS_PHASE = 256 * 4
SHT_REAL_NORM = 256 * 8
sht_gauss, sht_auto, sht_reg_fast, sht_reg_dct, sht_quick_init, sht_reg_poles, sht_gauss_fly = range(7)
SHT_NATIVE_LAYOUT = 0
SHT_THETA_CONTIGUOUS = 256
SHT_PHI_CONTIGUOUS = 256 * 2
SHT_SOUTH_POLE_FIRST = 256 * 32
SHT_SCALAR_ONLY = 256 * 16
SHT_LOAD_SAVE_CFG = 256 * 64
SHT_ALLOW_GPU = 256 * 128
SHT_ALLOW_PADDING = 256 * 256


class ShtnsInfo(C.Structure):
    """Public prefix of struct shtns_info (shtns.h:79-94)."""
    _fields_ = [
        ("nlm", C.c_uint), ("lmax", C.c_ushort), ("mmax", C.c_ushort), ("mres", C.c_ushort),
        ("nlat_2", C.c_ushort), ("nlat", C.c_uint), ("nphi", C.c_uint), ("nspat", C.c_uint),
        ("li", C.POINTER(C.c_ushort)), ("mi", C.POINTER(C.c_ushort)),
        ("ct", C.POINTER(C.c_double)), ("st", C.POINTER(C.c_double)),
        ("nlat_padded", C.c_uint), ("nlm_cplx", C.c_uint),
    ]


class CPLX(C.Structure):
    """C99 double complex returned by value (two doubles)."""
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


CFG = C.POINTER(ShtnsInfo)
P = C.c_void_p
I = C.c_int
D = C.c_double

# name -> (restype, argtypes); every symbol include/*.h declares
PROTOTYPES = {
    # shtns.h
    "nlm_calc": (C.c_long, [C.c_long, C.c_long, C.c_long]),
    "nlm_cplx_calc": (C.c_long, [C.c_long, C.c_long, C.c_long]),
    "shtns_verbose": (None, [I]),
    "shtns_print_version": (None, []),
    "shtns_get_build_info": (C.c_char_p, []),
    "shtns_print_cfg": (None, [CFG]),
    "shtns_init": (CFG, [I, I, I, I, I, I]),
    "shtns_create": (CFG, [I, I, I, I]),
    "shtns_set_grid": (I, [CFG, I, D, I, I]),
    "shtns_set_grid_auto": (I, [CFG, I, D, I, C.POINTER(I), C.POINTER(I)]),
    "shtns_create_with_grid": (CFG, [CFG, I, I]),
    "shtns_use_threads": (I, [I]),
    "shtns_use_gpu": (I, [I]),
    "shtns_reset": (None, []),
    "shtns_destroy": (None, [CFG]),
    "shtns_unset_grid": (None, [CFG]),
    "shtns_robert_form": (None, [CFG, I]),
    "shtns_malloc": (P, [C.c_size_t]),
    "shtns_free": (None, [P]),
    "sh00_1": (D, [CFG]),
    "sh10_ct": (D, [CFG]),
    "sh11_st": (D, [CFG]),
    "shlm_e1": (D, [CFG, I, I]),
    "shtns_gauss_wts": (I, [CFG, P]),
    "spat_to_SH": (None, [CFG, P, P]),
    "SH_to_spat": (None, [CFG, P, P]),
    "spat_to_SHsphtor": (None, [CFG, P, P, P, P]),
    "SHsphtor_to_spat": (None, [CFG, P, P, P, P]),
    "SHsph_to_spat": (None, [CFG, P, P, P]),
    "SHtor_to_spat": (None, [CFG, P, P, P]),
    "spat_to_SHqst": (None, [CFG, P, P, P, P, P, P]),
    "SHqst_to_spat": (None, [CFG, P, P, P, P, P, P]),
    "spat_to_SH_l": (None, [CFG, P, P, I]),
    "SH_to_spat_l": (None, [CFG, P, P, I]),
    "SHsphtor_to_spat_l": (None, [CFG, P, P, P, P, I]),
    "SHsph_to_spat_l": (None, [CFG, P, P, P, I]),
    "SHtor_to_spat_l": (None, [CFG, P, P, P, I]),
    "spat_to_SHsphtor_l": (None, [CFG, P, P, P, P, I]),
    "spat_to_SHqst_l": (None, [CFG, P, P, P, P, P, P, I]),
    "SHqst_to_spat_l": (None, [CFG, P, P, P, P, P, P, I]),
    # shtns_cuda.h
    "cu_spat_to_SH": (None, [CFG, P, P, I]),
    "cu_spat_to_SH_float": (None, [CFG, P, P, I]),
    "cu_SH_to_spat": (None, [CFG, P, P, I]),
    "cu_SH_to_spat_float": (None, [CFG, P, P, I]),
    "cu_spat_to_SHsphtor": (None, [CFG, P, P, P, P, I]),
    "cu_SHsphtor_to_spat": (None, [CFG, P, P, P, P, I]),
    "cu_spat_to_SHqst": (None, [CFG, P, P, P, P, P, P, I]),
    "cu_SHqst_to_spat": (None, [CFG, P, P, P, P, P, P, I]),
    "cushtns_clone": (CFG, [CFG, P, P]),
    "cushtns_init_gpu": (I, [CFG]),
    "cushtns_set_streams": (None, [CFG, P, P]),
    # shtns_b200.h
    "shtns_set_batch": (I, [CFG, I, C.c_long, C.c_long]),
    "shtns_b200_error_mode": (None, [I]),
    "shtns_b200_last_error": (C.c_char_p, []),
    "shtns_b200_status": (I, []),
    "shtns_b200_device": (I, [CFG]),
    "shtns_b200_device_bytes": (C.c_size_t, [CFG]),
    "shtns_b200_launch_count": (C.c_long, []),
    "shtns_b200_set_timing": (None, [CFG, I]),
    "shtns_b200_stage_times": (I, [CFG, P, P]),
    "shtns_b200_polar_rows": (I, [CFG, P]),
    "cu_SH_to_spat_noalloc": (None, [CFG, P, P, I]),
    "cu_SH_to_spat_adjoint": (None, [CFG, P, P, I]),
    "cu_spat_to_SH_adjoint": (None, [CFG, P, P, I]),
    "shtns_b200_set_option": (I, [CFG, I, I]),
    "SH_to_spat_cplx": (None, [CFG, P, P]),
    "spat_cplx_to_SH": (None, [CFG, P, P]),
    "SHsphtor_to_spat_cplx": (None, [CFG, P, P, P, P]),
    "spat_cplx_to_SHsphtor": (None, [CFG, P, P, P, P]),
    "SHqst_to_spat_cplx": (None, [CFG, P, P, P, P, P, P]),
    "spat_cplx_to_SHqst": (None, [CFG, P, P, P, P, P, P]),
    "SH_to_spat_ml": (None, [CFG, I, P, P, I]),
    "spat_to_SH_ml": (None, [CFG, I, P, P, I]),
    "SHsphtor_to_spat_ml": (None, [CFG, I, P, P, P, P, I]),
    "spat_to_SHsphtor_ml": (None, [CFG, I, P, P, P, P, I]),
    "SHsph_to_spat_ml": (None, [CFG, I, P, P, P, I]),
    "SHtor_to_spat_ml": (None, [CFG, I, P, P, P, I]),
    "SHqst_to_spat_ml": (None, [CFG, I, P, P, P, P, P, P, I]),
    "spat_to_SHqst_ml": (None, [CFG, I, P, P, P, P, P, P, I]),
    "shtns_b200_kernel_errors": (I, [CFG]),
    "shtns_b200_split_table_bytes": (C.c_size_t, [CFG]),
    "shtns_b200_get_option": (I, [CFG, I]),
    "shtns_b200_group_create": (P, [I, P]),
    "shtns_b200_group_destroy": (None, [P]),
    "shtns_b200_group_set_option": (I, [P, I, I]),
    "shtns_b200_group_synth": (None, [P, P, P, P, I]),
    "shtns_b200_group_analys": (None, [P, P, P, P, I]),
    "shtns_b200_group_SHsphtor_to_spat": (None, [P, P, P, P, P, P, I]),
    "shtns_b200_group_spat_to_SHsphtor": (None, [P, P, P, P, P, P, I]),
    "shtns_b200_group_SHqst_to_spat": (None, [P, P, P, P, P, P, P, P, I]),
    "shtns_b200_group_spat_to_SHqst": (None, [P, P, P, P, P, P, P, P, I]),
    "SH_to_point": (D, [CFG, P, D, D]),
    "SH_to_point_cplx": (CPLX, [CFG, P, D, D]),
    "SH_to_grad_point": (None, [CFG, P, P, D, D, P, P, P]),
    "SHqst_to_point": (None, [CFG, P, P, P, D, D, P, P, P]),
    "SH_to_lat": (None, [CFG, P, D, P, I, I, I]),
    "SHqst_to_lat": (None, [CFG, P, P, P, D, P, P, P, I, I, I]),
    "legendre_sphPlm_array": (I, [CFG, I, I, D, P]),
    "legendre_sphPlm_deriv_array": (I, [CFG, I, I, D, D, P, P]),
    "mul_ct_matrix": (None, [CFG, P]),
    "st_dt_matrix": (None, [CFG, P]),
    "SH_mul_mx": (None, [CFG, P, P, P]),
    "SH_Zrotate": (None, [CFG, P, D, P]),
    "SH_Yrotate": (None, [CFG, P, D, P]),
    "SH_Yrotate90": (None, [CFG, P, P]),
    "SH_Xrotate90": (None, [CFG, P, P]),
    "shtns_rotation_create": (P, [I, I, I]),
    "shtns_rotation_destroy": (None, [P]),
    "shtns_rotation_set_angles_ZYZ": (None, [P, D, D, D]),
    "shtns_rotation_set_angles_ZXZ": (None, [P, D, D, D]),
    "shtns_rotation_set_angle_axis": (None, [P, D, D, D, D]),
    "shtns_rotation_wigner_d_matrix": (I, [P, I, P]),
    "shtns_rotation_apply_cplx": (None, [P, P, P]),
    "shtns_rotation_apply_real": (None, [P, P, P]),
    "shtns_b200_SH_to_points": (None, [CFG, P, P, P, P, I]),
    "shtns_b200_SHqst_to_points": (None, [CFG, P, P, P, P, P, P, P, P, I]),
    "shtns_b200_legendre_synth_rows": (None, [CFG, I, P, P, P, I, I, I, I, P, P]),
    "shtns_b200_legendre_analys_rows": (None, [CFG, I, I, P, P, P, P, P, I, I, I]),
    "shtns_b200_alloc": (P, [C.c_size_t]),
    "shtns_b200_free": (None, [P]),
    "shtns_b200_ipc_handle": (I, [P, P]),
    "shtns_b200_ipc_open": (P, [P]),
    "shtns_b200_ipc_close": (None, [P]),
    "shtns_b200_legendre_synth": (None, [CFG, I, P, P, P, P, I, I, I]),
    "shtns_b200_fourier_synth": (None, [CFG, I, P, P, P, P, I, I]),
    "shtns_b200_fourier_analys": (None, [CFG, I, P, P, P, P, I, I]),
    "shtns_b200_legendre_analys": (None, [CFG, I, P, P, P, P, I, I, I]),
}

_lib = None


def load():
    """Load libshtns_b200.so and declare every prototype."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"shtns_b200 CUDA library not built: {LIB_PATH} missing "
                          "(run `python -m shtns_b200.build`)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib.shtns_b200_error_mode(1)     # Python callers get error returns instead of exit()
    _lib = lib
    return lib


class SHTError(RuntimeError):
    pass


def check(lib=None):
    """Raise SHTError if a transform error was recorded since the last check."""
    lib = lib or load()
    st = lib.shtns_b200_status()
    if st:
        raise SHTError(lib.shtns_b200_last_error().decode())
