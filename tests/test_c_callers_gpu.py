"""The drop-in boundary exercised from C, not only through ctypes.

* The reference's own known-answer program, examples/test_suite.c:96-152
  (analytic field at lmax=7 on 64 x 8, ftol 1e-14), compiled unchanged as C99
  against include/shtns.h and linked to libshtns_b200.so by oracle/Makefile
  (the reference sources exist only where the library is built, so the
  binary is prebuilt into oracle/_ref).
* tests/c/cu_roundtrip.c, a cudamaxrelerror.cu-style caller (the reference's
  cudamaxrelerror.cu:22-94): host transforms beside cu_* device transforms,
  compiled here with gcc -std=c99 against include/shtns.h + shtns_cuda.h.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def test_reference_test_suite_program_passes():
    exe = os.path.join(ROOT, "oracle", "_ref", "test_suite_b200")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/test_suite_b200 not built (needs the reference sources)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout, r.stdout


def test_c99_device_api_caller(tmp_path):
    exe = str(tmp_path / "cu_roundtrip")
    cmd = ["gcc", "-std=c99", "-D_DEFAULT_SOURCE", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "c", "cu_roundtrip.c"),
           "-L", os.path.join(ROOT, "shtns_b200"), "-lshtns_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-lm",
           "-Wl,-rpath," + os.path.join(ROOT, "shtns_b200"), "-o", exe]
    c = subprocess.run(cmd, capture_output=True, text=True)
    assert c.returncode == 0, c.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout, r.stdout
