"""Order-split CUDA stages on one GPU.  Several ranks are emulated in one
process: every rank's Legendre (or FFT) stage runs in turn, the all-to-all is
done by slicing the ranks' send buffers (no kernel waits on another), and the
assembled result is compared with the whole-field CUDA transform (same
kernels: expected equal to rounding) and with the oracle (1e-12)."""
import numpy as np
import pytest
import torch

from shtns_b200 import sht, SHT_THETA_CONTIGUOUS, SHT_PHI_CONTIGUOUS, sht_gauss
from shtns_b200.ordersplit import OrderSplit
from tests.common import rand_spec, relerr

pytestmark = pytest.mark.gpu


def _exchange(sends, world):
    """recv[d] = concatenation over sources s of chunk d of s's send buffer."""
    chunks = [torch.split(buf, sz) for buf, sz in sends]
    return [torch.cat([chunks[s][d] for s in range(world)]) for d in range(world)]


def emulated_synth(splits, specs, ltr=None):
    world = len(splits)
    F = [sp.synth_legendre(*specs, ltr=ltr) for sp in splits]
    recv = _exchange([sp.synth_send(f) for sp, f in zip(splits, F)], world)
    nfc = F[0].shape[0]
    blocks = [sp.synth_fourier(sp.synth_recv(r, nfc), specs[0].shape[:-1], len(specs), ltr)
              for sp, r in zip(splits, recv)]
    axis = -2 if splits[0].phi_contiguous else -1
    return [torch.cat([b[c] for b in blocks], dim=axis) for c in range(len(specs))]


def emulated_analys(splits, fields, ltr=None):
    world = len(splits)
    F = [sp.analys_fourier(*[sp.local_rows(v) for v in fields], ltr=ltr) for sp in splits]
    recv = _exchange([sp.analys_send(f) for sp, f in zip(splits, F)], world)
    nfc = F[0].shape[0]
    parts = [sp.analys_legendre(sp.analys_recv(r, nfc), fields[0].shape[:-2], len(fields), ltr)
             for sp, r in zip(splits, recv)]
    out = []
    for c in range(len(fields)):
        q = torch.zeros_like(parts[0][c])
        for sp, p in zip(splits, parts):
            sl = sp.spec_slice()
            q[..., sl] = p[c][..., sl]
        out.append(q)
    return out


def make_plan(lmax, mmax, mres, nlat, nphi, layout, eps=1e-10):
    s = sht(lmax, mmax, mres)
    s.set_grid(nlat, nphi, sht_gauss | layout, eps)
    return s


@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_order_split_scalar_matches_whole_transform(world):
    s = make_plan(127, 127, 1, 192, 384, SHT_PHI_CONTIGUOUS)
    q = torch.from_numpy(rand_spec(127, 127, 1, 5, nfields=3)).cuda()
    splits = [OrderSplit(s, rank=r, world=world) for r in range(world)]
    v = emulated_synth(splits, [q])[0]
    v_ref = s.synth(q)
    assert relerr(v_ref.cpu().numpy(), v.cpu().numpy()) < 1e-14
    qa = emulated_analys(splits, [v_ref])[0]
    qa_ref = s.analys(v_ref)
    assert relerr(qa_ref.cpu().numpy(), qa.cpu().numpy()) < 1e-14
    assert relerr(q.cpu().numpy(), qa.cpu().numpy()) < 1e-11


def test_order_split_single_process_call():
    s = make_plan(63, 63, 1, 96, 192, SHT_THETA_CONTIGUOUS)
    q = torch.from_numpy(rand_spec(63, 63, 1, 8)).cuda()
    sp = OrderSplit(s, rank=0, world=1)
    v = sp.synth(q)
    assert relerr(s.synth(q).cpu().numpy(), v.cpu().numpy()) < 1e-14
    assert relerr(q.cpu().numpy(), sp.analys(v).cpu().numpy()) < 1e-11


@pytest.mark.parametrize("layout", [SHT_THETA_CONTIGUOUS, SHT_PHI_CONTIGUOUS])
def test_order_split_vector_and_truncation(layout):
    lmax, mres, mmax = 95, 2, 40
    s = make_plan(lmax, mmax, mres, 144, 192, layout)
    rs = [torch.from_numpy(rand_spec(lmax, mmax, mres, 20 + i, nfields=2, zero_l0=(i > 0))).cuda()
          for i in range(3)]
    splits = [OrderSplit(s, rank=r, world=3) for r in range(3)]
    for ltr in (None, 60):
        got = emulated_synth(splits, rs, ltr=ltr)
        ref = s.synth(*rs, ltr=ltr)
        for a, b in zip(ref, got):
            assert relerr(a.cpu().numpy(), b.cpu().numpy()) < 1e-14
        got = emulated_analys(splits, list(ref), ltr=ltr)
        back = s.analys(*ref, ltr=ltr)
        for a, b in zip(back, got):
            assert relerr(a.cpu().numpy(), b.cpu().numpy()) < 1e-14
    # spheroidal/toroidal pair
    vt, vp = emulated_synth(splits, rs[1:])
    rt, rp = s.synth(*rs[1:])
    assert relerr(rt.cpu().numpy(), vt.cpu().numpy()) < 1e-14
    assert relerr(rp.cpu().numpy(), vp.cpu().numpy()) < 1e-14


def test_order_split_against_oracle():
    from oracle.sht_np import NpSHT
    lmax, nlat, nphi = 63, 96, 128
    s = make_plan(lmax, lmax, 1, nlat, nphi, SHT_PHI_CONTIGUOUS, eps=0.0)   # no polar threshold on either side
    qn = rand_spec(lmax, lmax, 1, 31, nfields=2)
    splits = [OrderSplit(s, rank=r, world=2) for r in range(2)]
    v = emulated_synth(splits, [torch.from_numpy(qn).cuda()])[0].cpu().numpy()
    ref = NpSHT(lmax, lmax, 1, 0, nlat, nphi, layout=SHT_PHI_CONTIGUOUS).synth(qn)
    assert relerr(ref, v) < 1e-12


def test_order_split_rejects_bad_ranges():
    from shtns_b200.capi import SHTError
    s = make_plan(31, 31, 1, 48, 64, SHT_PHI_CONTIGUOUS)
    q = torch.zeros(s.nlm, dtype=torch.complex128, device="cuda")
    F = torch.zeros((1, 32, 48), dtype=torch.complex128, device="cuda")
    st = OrderSplit(s, rank=0, world=1).stages
    with pytest.raises(SHTError):
        st.legendre_synth(0, [q], F, 5, 40, 31, 1)        # m1 > mmax
    with pytest.raises(SHTError):
        st.fourier_synth(0, F, [torch.zeros(3, 64, dtype=torch.float64, device="cuda")], 3, 31, 1)  # odd rows
    assert np.isfinite(F.cpu().numpy()).all()


def _fused_splits(s, world, nfc):
    from shtns_b200.ordersplit import FusedOrderSplit
    splits = [FusedOrderSplit(s, rank=r, world=world, barrier=lambda: None) for r in range(world)]
    for sp in splits:
        sp.allocate(nfc)
    ptrs = [sp.buf.ptr for sp in splits]
    for sp in splits:
        sp.set_row_buffers(ptrs)
    return splits


@pytest.mark.parametrize("world,layout,kind,nf", [(2, SHT_PHI_CONTIGUOUS, 1, 2), (3, SHT_THETA_CONTIGUOUS, 3, 2),
                                                  (4, SHT_PHI_CONTIGUOUS, 2, 2), (2, SHT_THETA_CONTIGUOUS, 1, 1)])
def test_fused_order_split_emulated_ranks(world, layout, kind, nf):
    """The exchange fused into the Legendre kernels: every emulated rank's
    synthesis stores its rows into all ranks' row buffers (local buffers
    here), each rank's FFT then reads its own; the analysis runs backwards.
    Same kernels as the whole transform: equal to rounding."""
    s = make_plan(127, 127, 1, 192, 256, layout)
    specs = [torch.from_numpy(rand_spec(127, 127, 1, 60 + i, nfields=nf, zero_l0=(kind > 1))).cuda()
             for i in range(kind)]
    if kind == 2:
        specs = specs[:2]
    n = len(specs)
    splits = _fused_splits(s, world, n * nf)
    for sp in splits:
        sp.synth_rows(*specs)
    blocks = [sp.synth_fourier(sp.own_rows(n * nf), specs[0].shape[:-1], n) for sp in splits]
    axis = -2 if splits[0].phi_contiguous else -1
    got = [torch.cat([b[c] for b in blocks], dim=axis) for c in range(n)]
    ref = s.synth(*specs)
    ref = list(ref) if isinstance(ref, tuple) else [ref]
    for a, b in zip(ref, got):
        assert relerr(a.cpu().numpy(), b.cpu().numpy()) < 1e-14
    for sp in splits:
        sp.analys_fourier_rows(*[sp.local_rows(v) for v in ref])
    parts = [sp.analys_rows(n, specs[0].shape[:-1], specs[0].device) for sp in splits]
    back = s.analys(*ref)
    back = list(back) if isinstance(back, tuple) else [back]
    for c in range(n):
        q = torch.zeros_like(back[c])
        for sp, p in zip(splits, parts):
            q[..., sp.spec_slice()] = p[c][..., sp.spec_slice()]
        assert relerr(back[c].cpu().numpy(), q.cpu().numpy()) < 1e-14
    for sp in splits:
        sp.release()


def test_fused_order_split_single_process_call():
    from shtns_b200.ordersplit import FusedOrderSplit
    s = make_plan(95, 95, 1, 144, 192, SHT_PHI_CONTIGUOUS)
    q = torch.from_numpy(rand_spec(95, 95, 1, 70, nfields=3)).cuda()
    sp = FusedOrderSplit(s, rank=0, world=1)
    v = sp.synth(q)
    assert relerr(s.synth(q).cpu().numpy(), v.cpu().numpy()) < 1e-14
    assert relerr(q.cpu().numpy(), sp.analys(v).cpu().numpy()) < 1e-11
    sp.release()
