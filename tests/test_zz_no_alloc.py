"""The allocation-free scalar synthesis, cu_SH_to_spat_noalloc.

It exists for callers that cannot call cudaMalloc where they transform (an
allocation-free region of a real-time loop or a plug-in host whose device
memory is owned by someone else): its scratch lives in a static device array
of the library instead of plan buffers grown on demand.  These tests call it
through the C ABI and compare it with cu_SH_to_spat, the entry point that
allocates, on two calls in a row, and check that it leaves the plan's device
memory untouched and rejects work larger than its static scratch.

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


def _plan(lmax, nlat, nphi):
    import shtns_b200
    sh = shtns_b200.sht(lmax)
    sh.set_grid(nlat, nphi, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=1e-10)
    return sh


def test_no_alloc_synthesis_matches_allocating_entry_point():
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    ref_plan = _plan(127, 192, 384)          # uses the allocating entry point
    na_plan = _plan(127, 192, 384)           # only ever used through the no-alloc entry point
    bytes_before = lib.shtns_b200_device_bytes(na_plan._cfg)
    lib.cushtns_set_streams(na_plan._cfg, C.c_void_p(torch.cuda.current_stream().cuda_stream), None)
    for seed in (11, 12):                    # two calls in a row, different inputs
        q = torch.from_numpy(rand_spec(127, 127, 1, seed)).to(dev)
        v_ref = ref_plan.synth(q)
        v = torch.full((384, 192), float("nan"), dtype=torch.float64, device=dev)
        lib.shtns_b200_status()
        lib.cu_SH_to_spat_noalloc(na_plan._cfg, C.c_void_p(q.data_ptr()), C.c_void_p(v.data_ptr()), 127)
        torch.cuda.synchronize()
        assert lib.shtns_b200_status() == 0, lib.shtns_b200_last_error().decode()
        a, b = v_ref.cpu().numpy(), v.cpu().numpy()
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
