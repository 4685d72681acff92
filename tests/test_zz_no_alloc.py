"""The allocation-free scalar synthesis, cu_SH_to_spat_noalloc.

It exists for callers that cannot call cudaMalloc where they transform (an
allocation-free region of a real-time loop or a plug-in host whose device
memory is owned by someone else): its scratch lives in a static device array
of the library instead of plan buffers grown on demand.  These tests call it
through the C ABI and compare it with cu_SH_to_spat, the entry point that
allocates, on two calls in a row, and check that it leaves the plan's device
memory untouched and rejects work larger than its static scratch.

Before every call the static array is filled with 0xFF bytes (NaN doubles)
through plan option 9, so a call that read scratch it had not written in the
same call would give NaN, not the previous call's (equal) values.

This file is collected last on purpose (pytest orders files by name), so a
run that stops at the first failure has run every other test first; it also
passes when run alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from tests.common import rand_spec, relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12
OPT_FILL_STATIC_SCRATCH = 9


def _plan(lmax, nlat, nphi, phi_contiguous=False):
    import shtns_b200
    sh = shtns_b200.sht(lmax)
    layout = 0 if phi_contiguous else shtns_b200.SHT_THETA_CONTIGUOUS
    sh.set_grid(nlat, nphi, flags=shtns_b200.sht_quick_init | layout, polar_opt=1e-10)
    return sh


# lmax, nlat, nphi, fields, ltr, phi-contiguous: one field (SIMT Legendre
# kernels), a truncated one, 8 fields (tensor-core tiles) and a
# phi-contiguous grid; every case fits the 32 MiB static scratch.
CASES = [(127, 192, 384, 1, 127, False), (127, 192, 384, 1, 80, False), (127, 192, 384, 8, 127, False),
         (95, 144, 288, 4, 60, True), (511, 768, 1536, 1, 511, False)]


@pytest.mark.parametrize("lmax,nlat,nphi,nf,ltr,phic", CASES)
def test_no_alloc_synthesis_matches_allocating_entry_point(lmax, nlat, nphi, nf, ltr, phic):
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    ref_plan = _plan(lmax, nlat, nphi, phic)          # uses the allocating entry point
    na_plan = _plan(lmax, nlat, nphi, phic)           # only ever used through the no-alloc entry point
    spat_shape = na_plan.spat_shape
    assert lib.shtns_set_batch(na_plan._cfg, nf, na_plan.nlm, na_plan.nspat) == 0
    bytes_before = lib.shtns_b200_device_bytes(na_plan._cfg)
    lib.cushtns_set_streams(na_plan._cfg, C.c_void_p(torch.cuda.current_stream().cuda_stream), None)
    for seed in (11, 12):                    # two calls in a row, different inputs
        q = torch.from_numpy(rand_spec(lmax, lmax, 1, seed, nfields=nf)).to(dev)
        v_ref = ref_plan.synth(q, ltr=ltr)
        v = torch.full((nf,) + spat_shape, float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        assert lib.shtns_b200_set_option(na_plan._cfg, OPT_FILL_STATIC_SCRATCH, 0xFF) == 0
        lib.shtns_b200_status()
        lib.cu_SH_to_spat_noalloc(na_plan._cfg, C.c_void_p(q.data_ptr()), C.c_void_p(v.data_ptr()), ltr)
        torch.cuda.synchronize()
        assert lib.shtns_b200_status() == 0, lib.shtns_b200_last_error().decode()
        a, b = v_ref.cpu().numpy().reshape(nf, -1), v.cpu().numpy().reshape(nf, -1)
        assert np.isfinite(b).all()
        assert relerr(a, b) < TOL
    # no work buffers were grown for the plan
    assert lib.shtns_b200_device_bytes(na_plan._cfg) == bytes_before


def test_no_alloc_rejects_work_beyond_the_static_scratch():
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    big = _plan(1023, 1536, 3072)            # one field needs about 58 MB of scratch
    q = torch.zeros(big.nlm, dtype=torch.complex128, device=dev)
    v = torch.zeros((3072, 1536), dtype=torch.float64, device=dev)
    lib.shtns_b200_status()
    lib.cu_SH_to_spat_noalloc(big._cfg, C.c_void_p(q.data_ptr()), C.c_void_p(v.data_ptr()), 1023)
    assert lib.shtns_b200_status() == 1
    assert "static" in lib.shtns_b200_last_error().decode()


def test_no_alloc_rejects_split_precision_plans():
    """A plan switched to split-precision synthesis (option 4) is refused with
    an error instead of silently computing the FP64 form."""
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    sh = _plan(127, 192, 384)
    assert lib.shtns_b200_set_option(sh._cfg, 4, 5) == 0
    q = torch.zeros(sh.nlm, dtype=torch.complex128, device=dev)
    v = torch.zeros((384, 192), dtype=torch.float64, device=dev)
    lib.shtns_b200_status()
    lib.cu_SH_to_spat_noalloc(sh._cfg, C.c_void_p(q.data_ptr()), C.c_void_p(v.data_ptr()), 127)
    assert lib.shtns_b200_status() == 1
    assert "split" in lib.shtns_b200_last_error().decode()
