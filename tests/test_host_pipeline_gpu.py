"""Host-pointer transforms (SH_to_spat, SHqst_to_spat, spat_to_SHqst, ... with
host arrays): the fields are pipelined in chunks over the transfer stream,
the compute stream and a second copy stream.  Checked against the device-
pointer transforms on the same inputs (the same kernels: equal to rounding),
for pageable NumPy arrays and for page-locked arrays from shtns_malloc, with
a batch whose last chunk is shorter than the others, and for one field."""
import ctypes as C

import numpy as np
import pytest

from tests.common import rand_spec, relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-14


def _plan(L=127, nlat=192, nphi=384):
    import shtns_b200
    sh = shtns_b200.sht(L)
    sh.set_grid(nlat, nphi, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=1e-10)
    return sh


def _pinned(lib, shape, dtype):
    """NumPy view of page-locked memory from shtns_malloc (freed by the caller)."""
    n = int(np.prod(shape)) * np.dtype(dtype).itemsize
    p = lib.shtns_malloc(n)
    assert p
    buf = (C.c_char * n).from_address(p)
    return np.frombuffer(buf, dtype=dtype).reshape(shape), p


@pytest.mark.parametrize("nf", [1, 20])
def test_host_pipeline_matches_device_api_pageable_and_pinned(nf):
    from shtns_b200 import capi
    lib = capi.load()
    L = 127
    sh = _plan(L)
    dev = torch.device("cuda:0")
    q = rand_spec(L, L, 1, 3, power=1.0, nfields=nf)
    s = rand_spec(L, L, 1, 4, power=1.5, zero_l0=True, nfields=nf)
    t = rand_spec(L, L, 1, 5, power=1.5, zero_l0=True, nfields=nf)
    # device-pointer reference
    dv = sh.synth(*(torch.from_numpy(a).to(dev) for a in (q, s, t)))
    dq = sh.analys(*dv)
    ref_v = [x.cpu().numpy() for x in dv]
    ref_q = [x.cpu().numpy() for x in dq]
    # pageable host arrays (NumPy) through the host API
    hv = sh.synth(q, s, t)
    hq = sh.analys(*ref_v)
    for a, b in zip(ref_v, hv):
        assert relerr(a, b) < TOL
    for a, b in zip(ref_q, hq):
        assert relerr(a, b) < TOL
    # page-locked arrays from shtns_malloc, C API directly
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    spec = [_pinned(lib, (nf, sh.nlm), np.complex128) for _ in range(3)]
    spat = [_pinned(lib, (nf,) + sh.spat_shape, np.float64) for _ in range(3)]
    back = [_pinned(lib, (nf, sh.nlm), np.complex128) for _ in range(3)]
    try:
        for (a, _), src in zip(spec, (q, s, t)):
            a[...] = src
        assert lib.shtns_set_batch(sh._cfg, nf, sh.nlm, sh.nspat) == 0
        lib.shtns_b200_status()
        lib.SHqst_to_spat(sh._cfg, *(P(a) for a, _ in spec), *(P(a) for a, _ in spat))
        lib.spat_to_SHqst(sh._cfg, *(P(a) for a, _ in spat), *(P(a) for a, _ in back))
        assert lib.shtns_b200_status() == 0, lib.shtns_b200_last_error().decode()
        for a, (b, _) in zip(ref_v, spat):
            assert relerr(a, b) < TOL
        for a, (b, _) in zip(ref_q, back):
            assert relerr(a, b) < TOL
    finally:
        for _, p in spec + spat + back:
            lib.shtns_free(C.c_void_p(p))


def test_host_pipeline_scalar_truncated_batch():
    """Scalar synthesis and analysis of 13 fields (chunks of 2, the last of 1)
    at ltr < lmax through SH_to_spat_l / spat_to_SH_l."""
    L = 127
    sh = _plan(L)
    dev = torch.device("cuda:0")
    q = rand_spec(L, L, 1, 8, nfields=13)
    ref = sh.synth(torch.from_numpy(q).to(dev), ltr=90).cpu().numpy()
    got = sh.synth(q, ltr=90)
    assert relerr(ref, got) < TOL
    ref_a = sh.analys(torch.from_numpy(ref).to(dev), ltr=90).cpu().numpy()
    got_a = sh.analys(ref, ltr=90)
    assert relerr(ref_a, got_a) < TOL
