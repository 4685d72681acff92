"""CPU checks of the C-ABI library: it loads, exports every symbol that
include/*.h declares, and its host-side plan logic (sizes, index arrays,
argument validation, error reporting) behaves like the reference's
shtns_create / shtns_set_grid without needing a GPU."""
import ctypes as C
import os
import re

import pytest

from shtns_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    for h in ("shtns.h", "shtns_cuda.h", "shtns_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//.*", "", text)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\([^;{]*\)\s*;", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "return", "sizeof"):
                names.add(name)
    return sorted(names)


def test_headers_declare_the_transform_api():
    names = header_functions()
    for must in ("shtns_create", "shtns_set_grid", "SH_to_spat", "spat_to_SH", "SHsphtor_to_spat",
                 "spat_to_SHsphtor", "SHqst_to_spat", "spat_to_SHqst", "cu_SH_to_spat", "cu_spat_to_SH",
                 "cu_SHsphtor_to_spat", "cu_spat_to_SHsphtor", "cu_SHqst_to_spat", "cu_spat_to_SHqst",
                 "cushtns_clone", "cushtns_set_streams", "shtns_set_batch"):
        assert must in names, must


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers the headers exactly
    assert set(header_functions()) == set(capi.PROTOTYPES)


def test_nlm_calc_matches_reference_formula():
    lib = capi.load()
    for lmax, mmax, mres in [(127, 127, 1), (511, 511, 1), (40, 16, 2), (31, 10, 3)]:
        ref = (mmax + 1) * (lmax + 1) - mres * mmax * (mmax + 1) // 2      # sht_init.c:98-102
        assert lib.nlm_calc(lmax, mmax, mres) == ref


def test_create_sets_public_fields_and_index_arrays():
    lib = capi.load()
    cfg = lib.shtns_create(40, 16, 2, capi.sht_orthonormal)
    assert cfg
    s = cfg.contents
    assert (s.lmax, s.mmax, s.mres) == (40, 16, 2)
    assert s.nlm == lib.nlm_calc(40, 16, 2)
    lm = 0
    for im in range(17):
        for l in range(2 * im, 41):
            assert s.li[lm] == l and s.mi[lm] == 2 * im
            lm += 1
    assert lm == s.nlm
    # LM macro of shtns.h:106
    def LM(l, m):
        return ((m // 2) * (2 * 40 + 2 - (m + 2))) // 2 + l
    assert s.li[LM(33, 10)] == 33 and s.mi[LM(33, 10)] == 10
    lib.shtns_destroy(cfg)


@pytest.mark.parametrize("args,msg", [
    ((1, 1, 1, 0), "lmax"),
    ((10, 11, 1, 0), "MMAX"),
    ((10, 5, 0, 0), "MRES"),
])
def test_create_rejects_invalid_sizes(args, msg):
    lib = capi.load()
    cfg = lib.shtns_create(*args)
    assert not cfg
    assert msg in lib.shtns_b200_last_error().decode()


def test_special_values_match_reference_conventions():
    import math
    lib = capi.load()
    cfg = lib.shtns_create(10, 10, 1, capi.sht_orthonormal)
    assert abs(lib.sh00_1(cfg) - math.sqrt(4 * math.pi)) < 1e-15          # sht_init.c:1190
    assert abs(lib.sh10_ct(cfg) - math.sqrt(4 * math.pi / 3)) < 1e-15
    assert abs(lib.sh11_st(cfg) + math.sqrt(2 * math.pi / 3)) < 1e-15     # CS phase
    lib.shtns_destroy(cfg)


def test_set_grid_rejects_invalid_grids_before_touching_the_gpu():
    lib = capi.load()
    cfg = lib.shtns_create(31, 31, 1, capi.sht_orthonormal)
    assert lib.shtns_set_grid(cfg, capi.sht_gauss, 0.0, 30, 64) == -1          # nlat <= lmax
    assert "Nlat" in lib.shtns_b200_last_error().decode()
    assert lib.shtns_set_grid(cfg, capi.sht_gauss, 0.0, 48, 62) == -1          # nphi <= 2 mmax
    assert lib.shtns_set_grid(cfg, capi.sht_gauss, 0.0, 47, 64) == -1          # odd nlat
    assert lib.shtns_set_grid(cfg, capi.sht_gauss, 0.0, 48, 11 * 7) == -1      # unsupported radix 11
    assert lib.shtns_set_grid(cfg, capi.sht_reg_fast, 0.0, 64, 64) == -1       # regular grids
    lib.shtns_destroy(cfg)


def test_transform_without_grid_reports_error():
    lib = capi.load()
    cfg = lib.shtns_create(10, 10, 1, capi.sht_orthonormal)
    lib.shtns_b200_status()
    lib.cu_SH_to_spat(cfg, None, None, 10)
    assert lib.shtns_b200_status() == 1
    lib.shtns_destroy(cfg)


def test_set_batch_validates():
    lib = capi.load()
    cfg = lib.shtns_create(10, 10, 1, capi.sht_orthonormal)
    assert lib.shtns_set_batch(cfg, 0, 0, 0) == -1
    assert lib.shtns_set_batch(cfg, 4, 0, 0) == 0
    lib.shtns_destroy(cfg)


def test_plan_options_validate_and_read_back():
    """shtns_b200_set_option accepts the documented values and rejects the
    others (return -1, nothing changed); shtns_b200_get_option reads back."""
    lib = capi.load()
    cfg = lib.shtns_create(31, 31, 1, capi.sht_orthonormal)
    cases = {
        1: ([0, 1, 2, 4, 8], [3, 16, -1]),          # latitude pairs per FFT CTA
        3: ([0, 1, 2, 3], [4, -1]),                 # FFT kernels
        4: ([0, 3, 5, 7], [1, 2, 8]),               # split-precision slices
        5: ([0, 1, 2, 4, 8], [3, 16]),              # Legendre tile shape
        7: ([0, 16, 4096], [8, 4112, -16]),         # test hook of the FFT wait
        8: ([0, 1], [2, -1]),                       # split-precision form
    }
    for opt, (good, bad) in cases.items():
        for v in good:
            assert lib.shtns_b200_set_option(cfg, opt, v) == 0, (opt, v)
            assert lib.shtns_b200_get_option(cfg, opt) == v, (opt, v)
        last = good[-1]
        for v in bad:
            assert lib.shtns_b200_set_option(cfg, opt, v) == -1, (opt, v)
            assert lib.shtns_b200_get_option(cfg, opt) == last, (opt, v)
    assert lib.shtns_b200_set_option(cfg, 99, 0) == -1
    assert lib.shtns_b200_get_option(cfg, 99) == -1
    lib.shtns_destroy(cfg)


def test_public_headers_compile_as_c99_and_cxx():
    """include/shtns.h, shtns_cuda.h and shtns_b200.h compile in a C99 unit
    (complex.h cplx, enums, extern "C" guards) and in a C++ unit, and the C
    caller of the device API (tests/c/cu_roundtrip.c) compiles and links
    against libshtns_b200.so with -Wall -Wextra -Werror.  Nothing is run."""
    import subprocess
    import tempfile
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    inc = os.path.join(root, "include")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    cuda_lib = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "lib64")
    src = ('#include "shtns.h"\n#include "shtns_cuda.h"\n#include "shtns_b200.h"\n'
           'int f(shtns_cfg s) { return (int) s->nlm + (int) sizeof(cplx) + sht_quick_init + SHT_ALLOW_GPU; }\n')
    with tempfile.TemporaryDirectory() as d:
        for lang, std in (("c", "-std=c99"), ("c++", "-std=c++17")):
            p = os.path.join(d, "h." + ("c" if lang == "c" else "cpp"))
            with open(p, "w") as f:
                f.write(src)
            r = subprocess.run(["gcc" if lang == "c" else "g++", std, "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                                "-I", inc, "-I", cuda_inc, p], capture_output=True, text=True)
            assert r.returncode == 0, r.stderr
        exe = os.path.join(d, "cu_roundtrip")
        r = subprocess.run(["gcc", "-std=c99", "-D_DEFAULT_SOURCE", "-Wall", "-Wextra", "-Werror", "-I", inc,
                            "-I", cuda_inc, os.path.join(root, "tests", "c", "cu_roundtrip.c"),
                            "-L", os.path.join(root, "shtns_b200"), "-lshtns_b200", "-L", cuda_lib, "-lcudart",
                            "-lm", "-o", exe], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
