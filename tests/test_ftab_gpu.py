"""FP64 Legendre synthesis from the precomputed table of Legendre values
(option 10 = 2, sht_ftab.cu) against the on-the-fly kernels (option 10 = 1) on
the same plans and inputs: the same products in the same order, so the
results agree bit for bit.  Cases: vector (qst) fields with a polar
threshold, a truncated call (ltr < lmax: coefficient rows beyond the call's
last step are zeros), a column tile that is not full, a grid whose half
latitude count is not a multiple of 32, and the automatic mode (option 10 =
0), which takes the table for these sizes; an mres = 2 plan, the adjoint of
the analysis (the same launch with row weights) and clones made before and
after the table is built (they use the base plan's table)."""
import numpy as np
import pytest

from tests.common import rand_spec

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _plan(L, nlat, nphi, eps):
    import shtns_b200
    sh = shtns_b200.sht(L)
    sh.set_grid(nlat, nphi, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=eps)
    return sh


def _both(sh, fn):
    from shtns_b200 import capi
    lib = capi.load()
    out = {}
    for mode in (1, 2, 0):
        assert lib.shtns_b200_set_option(sh._cfg, 10, mode) == 0
        assert lib.shtns_b200_get_option(sh._cfg, 10) == mode
        out[mode] = fn()
        assert sh.kernel_errors() == 0
    return out


@pytest.mark.parametrize("L,nlat,nphi,eps", [(255, 384, 768, 1e-10), (200, 304, 600, 0.0)])
def test_table_synthesis_bit_identical_qst(L, nlat, nphi, eps):
    dev = torch.device("cuda:0")
    sh = _plan(L, nlat, nphi, eps)
    nf = 7                                              # 21 field-components: the last column tile is partial
    q = torch.from_numpy(rand_spec(L, L, 1, 31, power=1.0, nfields=nf)).to(dev)
    s = torch.from_numpy(rand_spec(L, L, 1, 32, power=1.5, zero_l0=True, nfields=nf)).to(dev)
    t = torch.from_numpy(rand_spec(L, L, 1, 33, power=1.5, zero_l0=True, nfields=nf)).to(dev)
    out = _both(sh, lambda: sh.synth(q, s, t))
    for mode in (2, 0):
        for a, b in zip(out[mode], out[1]):
            assert torch.equal(a, b)


def test_table_synthesis_truncated_and_scalar():
    dev = torch.device("cuda:0")
    L = 255
    sh = _plan(L, 384, 768, 1e-10)
    q = torch.from_numpy(rand_spec(L, L, 1, 34, power=1.0, nfields=40)).to(dev)
    out = _both(sh, lambda: (sh.synth(q), sh.synth(q, ltr=170)))
    for mode in (2, 0):
        assert torch.equal(out[mode][0], out[1][0])
        assert torch.equal(out[mode][1], out[1][1])
    # the truncated synthesis is not the full one (the zero rows are really zero)
    assert not torch.equal(out[1][0], out[1][1])


def test_table_option_validation_and_round_trip():
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    L = 127
    sh = _plan(L, 192, 384, 1e-10)
    assert lib.shtns_b200_set_option(sh._cfg, 10, 3) == -1
    assert lib.shtns_b200_set_option(sh._cfg, 10, -1) == -1
    q = torch.from_numpy(rand_spec(L, L, 1, 35, power=1.0, nfields=24)).to(dev)
    assert lib.shtns_b200_set_option(sh._cfg, 10, 1) == 0
    sh.synth(q)                               # work buffers, no table
    b1 = lib.shtns_b200_device_bytes(sh._cfg)
    assert lib.shtns_b200_set_option(sh._cfg, 10, 2) == 0
    v = sh.synth(q)
    # the table built by this call counts in the plan's device memory, not in a clone's
    assert lib.shtns_b200_device_bytes(sh._cfg) > b1 + 1_000_000
    assert lib.shtns_b200_device_bytes(sh.clone()._cfg) < b1
    back = sh.analys(v)
    assert float((back - q).abs().max() / q.abs().max()) < 1e-12


def test_table_synthesis_mres2_adjoint_and_clones():
    """mres = 2 plan; the adjoint of the analysis (a synthesis with quadrature
    row weights, cu_spat_to_SH_adjoint); a clone built before the table
    exists and one built after share the base plan's table: all bit-identical
    to the on-the-fly kernels."""
    import ctypes as C
    import shtns_b200
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    L, M, mres = 255, 126, 2
    sh = shtns_b200.sht(L, M, mres)
    sh.set_grid(384, 768, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=1e-10)
    nf = 12
    q = torch.from_numpy(rand_spec(L, M, mres, 51, power=1.0, nfields=nf)).to(dev)
    early = sh.clone()                       # before the table is built
    out = {}
    for mode in (1, 2):
        for p in (sh, early):
            assert lib.shtns_b200_set_option(p._cfg, 10, mode) == 0
        out[mode] = sh.synth(q)
        out[mode, "early"] = early.synth(q)
        # adjoint of the analysis on the same coefficients
        adj = torch.empty((nf,) + sh.spat_shape, dtype=torch.float64, device=dev)
        sh._batch(nf)
        sh._stream()
        lib.cu_spat_to_SH_adjoint(sh._cfg, C.c_void_p(q.data_ptr()), C.c_void_p(adj.data_ptr()), L)
        capi.check(lib)
        out[mode, "adj"] = adj
        assert sh.kernel_errors() == 0 and early.kernel_errors() == 0
    late = sh.clone()                        # after the table exists
    assert lib.shtns_b200_set_option(late._cfg, 10, 2) == 0
    torch.cuda.synchronize()
    assert torch.equal(out[2], out[1])
    assert torch.equal(out[2, "early"], out[1])
    assert torch.equal(out[2, "adj"], out[1, "adj"])
    assert torch.equal(late.synth(q), out[1])
    assert late.kernel_errors() == 0
