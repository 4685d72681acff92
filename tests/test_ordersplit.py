"""Order-split transforms on CPU: the partition helpers, and the whole
exchange path (pack, torch.distributed all_to_all_single over gloo, unpack,
gather) with world sizes 2 and 3.  The four stages here are the NumPy oracle
(this machine has no GPU); test_ordersplit_gpu.py runs the same driver on the
CUDA stages."""
import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest
import torch.multiprocessing as mp

from shtns_b200.ordersplit import balanced_ranges, row_blocks

LMAX, NLAT, NPHI = 31, 48, 64


def test_balanced_ranges_cover_and_balance():
    rng = np.random.default_rng(3)
    for n in (3, 8, 32, 512):
        costs = np.arange(n, 0, -1) * 10 + rng.integers(0, 5, n)
        for w in (1, 2, 3, 8):
            if w > n:
                with pytest.raises(ValueError):
                    balanced_ranges(costs, w)
                continue
            rs = balanced_ranges(costs, w)
            assert rs[0][0] == 0 and rs[-1][1] == n - 1
            for (a, b), (c, _) in zip(rs, rs[1:]):
                assert b >= a and c == b + 1
            sums = [costs[a:b + 1].sum() for a, b in rs]
            # every part is within one order's cost of the ideal share
            assert max(sums) <= costs.sum() / w + costs.max()


def test_row_blocks_even_and_cover():
    for nlat in (4, 48, 770):
        for w in (1, 2, 3, 5):
            if nlat // 2 < w:
                continue
            bl = row_blocks(nlat, w)
            assert bl[0][0] == 0 and bl[-1][1] == nlat
            sizes = [b - a for a, b in bl]
            assert all(s % 2 == 0 and s > 0 for s in sizes)
            assert max(sizes) - min(sizes) <= 2
    with pytest.raises(ValueError):
        row_blocks(4, 3)


class OracleStages:
    """The four stages of a scalar transform computed by the NumPy oracle, on
    CPU torch tensors (same buffer layouts as the CUDA entry points)."""

    def __init__(self, sh, phi_contiguous):
        self.sh, self.phi = sh, phi_contiguous

    def legendre_synth(self, kind, specs, F, m0, m1, ltr, nf):
        assert kind == 0
        sh = self.sh
        q = specs[0].numpy().reshape(nf, sh.nlm)
        C = {}
        for im in range(m0, min(m1, ltr // sh.mres, sh.mmax) + 1):
            m, o = im * sh.mres, sh.m_offset(im)
            c = q[:, o:o + ltr - m + 1].copy()
            if m == 0:
                c = c.real.astype(np.complex128)
            C[im] = c
        if C:
            Fo = sh._legendre_synth(C, sh.lmax, ltr, False)      # [nf, nlat, mmax_t+1]
            for im in C:
                F[:, im - m0, :] = torch_from(Fo[:, :, im])

    def fourier_synth(self, kind, F, outs, nrows, ltr, nf):
        sh = self.sh
        ml = min(sh.mmax, ltr // sh.mres)
        G = np.zeros((nf, nrows, sh.nphi // 2 + 1), dtype=np.complex128)
        G[:, :, :ml + 1] = np.swapaxes(F.numpy()[:, :ml + 1, :], 1, 2)
        g = np.fft.irfft(G, n=sh.nphi, axis=-1) * sh.nphi
        if not self.phi:
            g = np.swapaxes(g, 1, 2)
        outs[0].copy_(torch_from(np.ascontiguousarray(g)).reshape(outs[0].shape))

    def fourier_analys(self, kind, ins, F, nrows, ltr, nf):
        sh = self.sh
        g = ins[0].numpy().reshape((nf,) + tuple(ins[0].shape[-2:]))
        if not self.phi:
            g = np.swapaxes(g, 1, 2)
        G = np.fft.rfft(g, axis=-1) / sh.nphi
        F.copy_(torch_from(np.ascontiguousarray(np.swapaxes(G[:, :, :sh.mmax + 1], 1, 2))))

    def legendre_analys(self, kind, F, outs, m0, m1, ltr, nf):
        sh = self.sh
        G = np.zeros((nf, sh.nlat, m1 + 1), dtype=np.complex128)
        G[:, :, m0:] = np.swapaxes(F.numpy(), 1, 2)
        Q = sh._legendre_analys(G, sh.lmax, ltr, False)
        out = outs[0].numpy().reshape(nf, sh.nlm)
        for im, c in Q.items():
            if im >= m0:
                o = sh.m_offset(im)
                out[:, o:o + c.shape[-1]] = c


def torch_from(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, layout, q, out):
    import torch
    import torch.distributed as dist
    from oracle.sht_np import NpSHT, SHT_PHI_CONTIGUOUS
    from shtns_b200.ordersplit import OrderSplit
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = NpSHT(LMAX, LMAX, 1, 0, NLAT, NPHI, layout=layout)
        plan = SimpleNamespace(lmax=LMAX, mmax=LMAX, mres=1, nlm=sh.nlm, nlat=NLAT, nphi=NPHI, layout=layout)
        phi = bool(layout & SHT_PHI_CONTIGUOUS)
        costs = np.arange(LMAX + 1, 0, -1)
        split = OrderSplit(plan, stages=OracleStages(sh, phi), costs=costs)
        qt = torch.from_numpy(q)
        v = split.synth(qt)                           # this rank's rows
        vfull = split.gather_spatial(v)
        qa = split.analys(split.local_rows(vfull))    # this rank's orders
        qfull = split.gather_spectral(qa)
        # truncated transform through the same exchange
        vt = split.gather_spatial(split.synth(qt, ltr=20))
        if rank == 0:
            out.put((vfull.numpy(), qfull.numpy(), vt.numpy(), split.orders, split.rows))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,layout", [(2, 512), (3, 256)])
def test_order_split_exchange_matches_single_process(world, layout):
    from oracle.sht_np import NpSHT
    from tests.common import rand_spec, relerr
    q = rand_spec(LMAX, LMAX, 1, 11, nfields=2)
    sh = NpSHT(LMAX, LMAX, 1, 0, NLAT, NPHI, layout=layout)
    v_ref = sh.synth(q)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, layout, q, out)) for r in range(world)]
    for p in procs:
        p.start()
    v, qa, vt, orders, rows = out.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert len(orders) == world and len(rows) == world
    assert relerr(v_ref, v) < 1e-14
    assert relerr(sh.analys(v_ref), qa) < 1e-14
    assert relerr(q, qa) < 1e-12                      # round trip
    assert relerr(sh.synth(q, ltr=20), vt) < 1e-14


class FakeLib:
    """Stand-in for the CUDA library's buffer and IPC entry points: pointers
    are integers, a handle encodes (rank, pointer), opening a peer's handle
    returns a pointer tagged with that peer."""

    def __init__(self, rank):
        self.rank = rank
        self.next = 0x1000 * (rank + 1)
        self.opened, self.closed, self.freed = [], [], []

    def shtns_b200_alloc(self, nbytes):
        self.next += 0x100
        return self.next

    def shtns_b200_free(self, p):
        self.freed.append(p.value)

    def shtns_b200_ipc_handle(self, p, h):
        data = ("%d:%d" % (self.rank, p.value)).encode().ljust(64, b"\0")
        for i, b in enumerate(data):
            h[i] = bytes([b])
        return 0

    def shtns_b200_ipc_open(self, h):
        r, ptr = h.value.decode().split(":")
        p = 0x7000000 + 0x1000 * int(r) + int(ptr)
        self.opened.append(p)
        return p

    def shtns_b200_ipc_close(self, p):
        self.closed.append(p.value)

    def shtns_b200_status(self):
        return 0


def _fused_worker(rank, world, port, out):
    import torch.distributed as dist
    from shtns_b200.ordersplit import FusedOrderSplit
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lib = FakeLib(rank)
        plan = SimpleNamespace(lmax=LMAX, mmax=LMAX, mres=1, nlm=528, nlat=NLAT, nphi=NPHI, layout=512, _lib=lib)
        sp = FusedOrderSplit(plan, costs=np.arange(LMAX + 1, 0, -1))
        sp.prepare(3)
        ptrs = list(sp.ptrs)
        bounds = list(sp.bounds)
        own = sp.buf.ptr
        sp.prepare(2)                      # large enough already: no new exchange
        again = list(sp.ptrs)
        sp.release()
        out.put((rank, own, ptrs, again, bounds, lib.opened, lib.closed, lib.freed))
    finally:
        dist.destroy_process_group()


def test_fused_split_maps_every_ranks_buffer_in_rank_order():
    world = 3
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fused_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owns = [r[1] for r in res]
    for rank, own, ptrs, again, bounds, opened, closed, freed in res:
        assert ptrs == again
        assert bounds[0] == 0 and bounds[-1] == NLAT and len(bounds) == world + 1
        for r, p in enumerate(ptrs):
            assert p == (own if r == rank else 0x7000000 + 0x1000 * r + owns[r])
        assert sorted(opened) == sorted(closed) and len(opened) == world - 1
        assert freed == [own]
