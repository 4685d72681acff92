"""CPU checks of the module-level part of the Python surface: the constants
and free functions that the reference's Python module exposes from shtns.h
(shtns_numpy.i:115-135), with the reference's names."""
import shtns_b200


def test_module_exposes_reference_names():
    for name in ("sht", "rotation", "nlm_calc", "nlm_cplx_calc", "set_verbosity", "print_version", "build_info",
                 "shtns_use_threads", "shtns_use_gpu",
                 "sht_orthonormal", "sht_fourpi", "sht_schmidt", "SHT_NO_CS_PHASE", "SHT_REAL_NORM",
                 "sht_gauss", "sht_auto", "sht_reg_fast", "sht_reg_dct", "sht_quick_init", "sht_reg_poles",
                 "sht_gauss_fly", "SHT_NATIVE_LAYOUT", "SHT_THETA_CONTIGUOUS", "SHT_PHI_CONTIGUOUS",
                 "SHT_SOUTH_POLE_FIRST", "SHT_SCALAR_ONLY", "SHT_LOAD_SAVE_CFG", "SHT_ALLOW_GPU", "SHT_ALLOW_PADDING"):
        assert hasattr(shtns_b200, name), name
    # enum values as in shtns.h:48-75
    assert (shtns_b200.sht_gauss, shtns_b200.sht_reg_fast, shtns_b200.sht_gauss_fly) == (0, 2, 6)
    assert shtns_b200.SHT_PHI_CONTIGUOUS == 512 and shtns_b200.SHT_ALLOW_PADDING == 65536


def test_module_functions():
    for lmax, mmax, mres in [(127, 127, 1), (40, 16, 2), (31, 10, 3)]:
        assert shtns_b200.nlm_calc(lmax, mmax, mres) == (mmax + 1) * (lmax + 1) - mres * mmax * (mmax + 1) // 2
    # complex fields: orders -mmax..mmax, (lmax+1)^2 for a full triangle
    assert shtns_b200.nlm_cplx_calc(10, 10, 1) == 121
    assert "SHTns" in shtns_b200.build_info()
    shtns_b200.set_verbosity(0)
    shtns_b200.print_version()
