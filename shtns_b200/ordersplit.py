"""One transform divided over processes by order m (one GPU per process).

The Legendre stage is independent per order and the phi FFT per grid row, so
one field too large for a single GPU's time budget is split this way:

* every rank owns a contiguous range of orders whose Legendre work (the sum
  over its orders of degrees x grid rows kept by the polar threshold) is about
  1/world of the total, and a block of consecutive grid rows (even counts that
  differ by at most two);
* synthesis: Legendre stage of the rank's orders over every row, one
  all-to-all that sends each rank the rows of its block, FFT of the block;
* analysis: FFT of the rank's block, the all-to-all backwards, Legendre stage
  of the rank's orders.

The reference transforms a field inside one process (sht_com.c:26-126,
sht_gpu.cu:584-1489); this split and its C entry points
(shtns_b200_legendre_synth / fourier_synth / fourier_analys /
legendre_analys) belong to this library.  The exchange is
torch.distributed.all_to_all_single (NCCL between GPUs).  Each phase is also a
public method, so a caller can run its own exchange between them.

Layouts on rank r: spectral arrays have the plan's full shape (..., nlm); the
synthesis reads only the rank's orders and the analysis writes them (other
orders zero; gather_spectral assembles the full array).  Spatial blocks are
grid rows lat0..lat1-1 in the plan's layout: (..., nrows, nphi) for a
phi-contiguous plan, (..., nphi, nrows) for a theta-contiguous one.
"""
import ctypes as C

import numpy as np

from . import capi

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None


def balanced_ranges(costs, world):
    """Split indices 0..len(costs)-1 into `world` contiguous, non-empty ranges
    (first, last) whose cost sums are as close as possible to total/world."""
    n = len(costs)
    if world < 1 or n < world:
        raise ValueError("need at least one order per rank")
    c = np.cumsum(np.asarray(costs, dtype=np.float64))
    total = c[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        i = int(np.searchsorted(c, target))          # c[i] >= target
        below = c[i - 1] if i > 0 else 0.0
        cut = i + 1 if (i < n and c[i] - target < target - below) else i
        cut = max(cut, cuts[-1] + 1)                 # non-empty
        cut = min(cut, n - (world - r))              # one index left for each later rank
        cuts.append(cut)
    cuts.append(n)
    return [(cuts[r], cuts[r + 1] - 1) for r in range(world)]


def row_blocks(nlat, world):
    """Blocks [lat0, lat1) of consecutive grid rows, even sizes differing by at
    most 2 (the FFT transforms rows in pairs)."""
    npair = nlat // 2
    if world < 1 or npair < world:
        raise ValueError("need at least one pair of grid rows per rank")
    base, extra = divmod(npair, world)
    out, a = [], 0
    for r in range(world):
        b = a + base + (1 if r < extra else 0)
        out.append((2 * a, 2 * b))
        a = b
    return out


def order_costs(plan):
    """Legendre work of each order index: degrees times grid rows kept by the
    polar threshold (shtns_b200_polar_rows)."""
    tm = (C.c_int * (plan.mmax + 1))()
    plan._lib.shtns_b200_polar_rows(plan._cfg, tm)
    im = np.arange(plan.mmax + 1)
    nl = plan.lmax + 1 - im * plan.mres
    rows = plan.nlat // 2 - np.asarray(tm[:], dtype=np.int64)
    return nl * np.maximum(rows, 1)


def lm_first(plan, im):
    """Index of (l = m, m = im*mres) in the spectral layout (shtns.h:104-106)."""
    return (im * (2 * plan.lmax + 2 - (im + 1) * plan.mres)) // 2 + im * plan.mres


class CudaStages:
    """The four order-split stages of the CUDA library on torch CUDA tensors,
    enqueued on torch's current stream."""

    def __init__(self, plan):
        self.plan = plan
        self.lib = plan._lib

    def _prep(self, nf):
        self.plan._batch(nf)
        self.plan._stream()

    @staticmethod
    def _ptrs(kind, arrs):
        p = [C.c_void_p(a.data_ptr()) for a in arrs]
        if kind == 0:
            return [p[0], None, None]
        if kind == 1:
            return [None, p[0], p[1]]
        return p

    @staticmethod
    def _vptrs(arrs):
        p = [C.c_void_p(a.data_ptr()) for a in arrs]
        return p + [None] * (3 - len(p))

    def legendre_synth(self, kind, specs, F, m0, m1, ltr, nf):
        self._prep(nf)
        q = self._ptrs(kind, specs)
        self.lib.shtns_b200_legendre_synth(self.plan._cfg, kind, q[0], q[1], q[2],
                                           C.c_void_p(F.data_ptr()), m0, m1, ltr)
        capi.check(self.lib)

    def fourier_synth(self, kind, F, outs, nrows, ltr, nf):
        self._prep(nf)
        v = self._vptrs(outs)
        self.lib.shtns_b200_fourier_synth(self.plan._cfg, kind, C.c_void_p(F.data_ptr()),
                                          v[0], v[1], v[2], nrows, ltr)
        capi.check(self.lib)

    def fourier_analys(self, kind, ins, F, nrows, ltr, nf):
        self._prep(nf)
        v = self._vptrs(ins)
        self.lib.shtns_b200_fourier_analys(self.plan._cfg, kind, v[0], v[1], v[2],
                                           C.c_void_p(F.data_ptr()), nrows, ltr)
        capi.check(self.lib)

    def legendre_analys(self, kind, F, outs, m0, m1, ltr, nf):
        self._prep(nf)
        q = self._ptrs(kind, outs)
        self.lib.shtns_b200_legendre_analys(self.plan._cfg, kind, C.c_void_p(F.data_ptr()),
                                            q[0], q[1], q[2], m0, m1, ltr)
        capi.check(self.lib)


class OrderSplit:
    """One transform of `plan` divided over the ranks of a process group by
    order.  rank/world default to the process group's; `stages` defaults to
    the CUDA library (tests may substitute another implementation of the four
    stages)."""

    def __init__(self, plan, group=None, rank=None, world=None, stages=None, costs=None):
        if plan.nlat == 0:
            raise RuntimeError("Grid not set. Call .set_grid() method.")
        if rank is None or world is None:
            import torch.distributed as dist
            rank = dist.get_rank(group) if rank is None else rank
            world = dist.get_world_size(group) if world is None else world
        if not (0 <= rank < world):
            raise ValueError("invalid rank/world")
        self.plan, self.group, self.rank, self.world = plan, group, rank, world
        self.stages = stages if stages is not None else CudaStages(plan)
        if costs is None:
            costs = order_costs(plan)
        self.orders = balanced_ranges(costs, world)   # (first, last) order index per rank
        self.rows = row_blocks(plan.nlat, world)      # [lat0, lat1) per rank
        self.m0, self.m1 = self.orders[rank]
        self.lat0, self.lat1 = self.rows[rank]
        self.nrows = self.lat1 - self.lat0
        self.nm = self.m1 - self.m0 + 1
        self.phi_contiguous = bool(plan.layout & capi.SHT_PHI_CONTIGUOUS)

    # ---------------- shapes ----------------
    def block_shape(self, r=None):
        n = self.nrows if r is None else self.rows[r][1] - self.rows[r][0]
        return (n, self.plan.nphi) if self.phi_contiguous else (self.plan.nphi, n)

    def spec_slice(self, r=None):
        """Slice of the spectral layout holding the orders of rank r."""
        a, b = self.orders[self.rank if r is None else r]
        return slice(lm_first(self.plan, a), lm_first(self.plan, b + 1))

    def local_rows(self, v):
        """This rank's block of a full spatial array (..., *spat_shape)."""
        if self.phi_contiguous:
            return v[..., self.lat0:self.lat1, :].contiguous()
        return v[..., :, self.lat0:self.lat1].contiguous()

    def _kind(self, n):
        if n not in (1, 2, 3):
            raise RuntimeError("1,2 or 3 arguments required.")
        return {1: 0, 2: 1, 3: 2}[n]

    def _ltr(self, ltr):
        return self.plan.lmax if ltr is None else int(ltr)

    # ---------------- synthesis phases ----------------
    def synth_legendre(self, *specs, ltr=None):
        """Legendre stage of this rank's orders: Fourier rows (nfc, nm, nlat)."""
        kind = self._kind(len(specs))
        specs = [s.contiguous() for s in specs]
        for s in specs:
            if s.dtype != torch.complex128 or s.shape[-1] != self.plan.nlm or s.shape != specs[0].shape:
                raise RuntimeError("spectral tensors must be complex128 (..., nlm) of one shape")
        nf = specs[0].numel() // self.plan.nlm
        F = torch.empty((len(specs) * nf, self.nm, self.plan.nlat), dtype=torch.complex128, device=specs[0].device)
        self.stages.legendre_synth(kind, specs, F, self.m0, self.m1, self._ltr(ltr), nf)
        return F

    def synth_send(self, F):
        """Pack the rows of every rank's block: (flat send buffer, split sizes)."""
        parts = [F[:, :, a:b].reshape(-1) for (a, b) in self.rows]
        return torch.cat(parts), [p.numel() for p in parts]

    def synth_recv_splits(self, nfc):
        return [nfc * (b - a + 1) * self.nrows for (a, b) in self.orders]

    def synth_recv(self, recv, nfc):
        """Unpack the received rows into (nfc, mmax+1, nrows)."""
        chunks = torch.split(recv, self.synth_recv_splits(nfc))
        return torch.cat([c.view(nfc, b - a + 1, self.nrows) for c, (a, b) in zip(chunks, self.orders)], dim=1)

    def synth_fourier(self, F, lead, n, ltr=None):
        """FFT of this rank's block: n spatial blocks (*lead, *block_shape)."""
        nf = F.shape[0] // n
        outs = [torch.empty(tuple(lead) + self.block_shape(), dtype=torch.float64, device=F.device)
                for _ in range(n)]
        self.stages.fourier_synth(self._kind(n), F, outs, self.nrows, self._ltr(ltr), nf)
        return outs

    def synth(self, *specs, ltr=None):
        """v = synth(qlm); vt, vp = synth(slm, tlm); vr, vt, vp = synth(qlm, slm,
        tlm), each the rank's block of grid rows (every rank calls it)."""
        F = self.synth_legendre(*specs, ltr=ltr)
        send, sin = self.synth_send(F)
        recv = self._exchange(send, sin, self.synth_recv_splits(F.shape[0]))
        outs = self.synth_fourier(self.synth_recv(recv, F.shape[0]), specs[0].shape[:-1], len(specs), ltr)
        return outs[0] if len(outs) == 1 else tuple(outs)

    # ---------------- analysis phases ----------------
    def analys_fourier(self, *blocks, ltr=None):
        """FFT of this rank's block: Fourier rows (nfc, mmax+1, nrows)."""
        kind = self._kind(len(blocks))
        blocks = [b.contiguous() for b in blocks]
        bs = self.block_shape()
        for b in blocks:
            if b.dtype != torch.float64 or tuple(b.shape[-2:]) != bs or b.shape != blocks[0].shape:
                raise RuntimeError("spatial blocks must be float64 (..., %d, %d) of one shape" % bs)
        nf = blocks[0].numel() // (bs[0] * bs[1])
        F = torch.empty((len(blocks) * nf, self.plan.mmax + 1, self.nrows), dtype=torch.complex128,
                        device=blocks[0].device)
        self.stages.fourier_analys(kind, blocks, F, self.nrows, self._ltr(ltr), nf)
        return F

    def analys_send(self, F):
        parts = [F[:, a:b + 1, :].reshape(-1) for (a, b) in self.orders]
        return torch.cat(parts), [p.numel() for p in parts]

    def analys_recv_splits(self, nfc):
        return [nfc * self.nm * (b - a) for (a, b) in self.rows]

    def analys_recv(self, recv, nfc):
        """Unpack into this rank's orders over every row: (nfc, nm, nlat)."""
        chunks = torch.split(recv, self.analys_recv_splits(nfc))
        return torch.cat([c.view(nfc, self.nm, b - a) for c, (a, b) in zip(chunks, self.rows)], dim=2)

    def analys_legendre(self, F, lead, n, ltr=None):
        """Legendre stage of this rank's orders: n spectral arrays (*lead, nlm)
        with the other orders zero."""
        nf = F.shape[0] // n
        outs = [torch.zeros(tuple(lead) + (self.plan.nlm,), dtype=torch.complex128, device=F.device)
                for _ in range(n)]
        self.stages.legendre_analys(self._kind(n), F, outs, self.m0, self.m1, self._ltr(ltr), nf)
        return outs

    def analys(self, *blocks, ltr=None):
        """qlm = analys(v); slm, tlm = analys(vt, vp); qlm, slm, tlm =
        analys(vr, vt, vp) from the rank's blocks of grid rows; the results
        hold this rank's orders (every rank calls it)."""
        F = self.analys_fourier(*blocks, ltr=ltr)
        send, sin = self.analys_send(F)
        recv = self._exchange(send, sin, self.analys_recv_splits(F.shape[0]))
        outs = self.analys_legendre(self.analys_recv(recv, F.shape[0]), blocks[0].shape[:-2], len(blocks), ltr)
        return outs[0] if len(outs) == 1 else tuple(outs)

    # ---------------- communication ----------------
    def _exchange(self, send, in_splits, out_splits):
        recv = torch.empty(sum(out_splits), dtype=send.dtype, device=send.device)
        if self.world == 1:
            recv.copy_(send)
            return recv
        import torch.distributed as dist
        dist.all_to_all_single(torch.view_as_real(recv), torch.view_as_real(send),
                               output_split_sizes=out_splits, input_split_sizes=in_splits, group=self.group)
        return recv

    def _gather_padded(self, local, sizes, dim):
        import torch.distributed as dist
        if self.world == 1:
            return local
        per = max(sizes)
        shape = list(local.shape)
        shape[dim] = per
        pad = torch.zeros(shape, dtype=local.dtype, device=local.device)
        pad.narrow(dim, 0, local.shape[dim]).copy_(local)
        parts = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(parts, pad, group=self.group)
        return torch.cat([p.narrow(dim, 0, n) for p, n in zip(parts, sizes)], dim=dim)

    def gather_spectral(self, q):
        """Full spectral arrays on every rank from each rank's orders."""
        sl = [self.spec_slice(r) for r in range(self.world)]
        sizes = [s.stop - s.start for s in sl]
        local = q[..., self.spec_slice()].contiguous()
        if q.is_complex():
            return torch.view_as_complex(self._gather_padded(torch.view_as_real(local), sizes, local.dim() - 1)
                                         .contiguous())
        return self._gather_padded(local, sizes, local.dim() - 1)

    def gather_spatial(self, v):
        """Full spatial arrays on every rank from each rank's block of rows."""
        sizes = [b - a for (a, b) in self.rows]
        return self._gather_padded(v.contiguous(), sizes, v.dim() - (2 if self.phi_contiguous else 1))


class RowBuffer:
    """A device allocation of its own holding one rank's Fourier rows
    [fc][order][row] (complex128), visible to torch through
    __cuda_array_interface__ without a copy."""

    def __init__(self, lib, shape):
        self.lib = lib
        self.shape = tuple(int(x) for x in shape)
        nbytes = 16 * int(np.prod(self.shape))
        self.ptr = lib.shtns_b200_alloc(nbytes)
        if not self.ptr:
            capi.check(lib)
            raise MemoryError("device buffer of %d bytes" % nbytes)
        self.__cuda_array_interface__ = {"shape": self.shape, "typestr": "<c16", "data": (self.ptr, False),
                                         "version": 3, "strides": None}

    def tensor(self):
        return torch.as_tensor(self, device=torch.device("cuda", torch.cuda.current_device()))

    def free(self):
        if self.ptr:
            self.lib.shtns_b200_free(C.c_void_p(self.ptr))
            self.ptr = None


class FusedOrderSplit(OrderSplit):
    """OrderSplit with the all-to-all fused into the Legendre kernels: the
    synthesis stores every Fourier row straight into the row buffer of the
    rank that owns the row (another GPU's memory mapped by CUDA IPC, over
    NVLink), the analysis loads rows from there, and the FFT stages work on
    the rank's own buffer.  Each direction runs
        barrier, Legendre stage into / from the buffers, barrier, FFT stage
    (synthesis), or FFT, barrier, Legendre, barrier (analysis): the barriers
    order the writes of one rank's kernels before the reads of another's.
    Each barrier first waits on the host for the rank's own work on torch's
    current stream (the stream the stages are enqueued on), then meets the
    other ranks: a rank's kernels, and so its peer stores, have completed
    before any other rank passes the barrier and launches kernels that read
    them, whatever the backend's barrier does with streams.
    Buffers are allocated and mapped by prepare(nfc), a collective call."""

    def __init__(self, plan, group=None, rank=None, world=None, costs=None, barrier=None):
        super().__init__(plan, group=group, rank=rank, world=world, costs=costs)
        self.lib = plan._lib
        self.buf = None
        self.ptrs = None
        self._mapped = []
        self._barrier = barrier

    def barrier(self):
        import torch
        if torch.cuda.is_available():
            torch.cuda.current_stream().synchronize()
        if self._barrier is not None:
            self._barrier()
        elif self.world > 1:
            import torch.distributed as dist
            dist.barrier(group=self.group)

    def release(self):
        for p in self._mapped:
            self.lib.shtns_b200_ipc_close(C.c_void_p(p))
        self._mapped = []
        if self.buf is not None:
            self.buf.free()
            self.buf = None
        self.ptrs = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def prepare(self, nfc):
        """Row buffer for nfc field-components on every rank, mapped into
        every rank (collective; nothing to do when the buffers are large enough)."""
        if self.buf is not None and self.buf.shape[0] >= nfc:
            return
        self.allocate(nfc)
        if self.world == 1:
            self.set_row_buffers([self.buf.ptr])
            return
        import torch.distributed as dist
        h = (C.c_char * 64)()
        if self.lib.shtns_b200_ipc_handle(C.c_void_p(self.buf.ptr), h) != 0:
            capi.check(self.lib)
        hs = [None] * self.world
        dist.all_gather_object(hs, bytes(h), group=self.group)
        ptrs = []
        for r, hb in enumerate(hs):
            if r == self.rank:
                ptrs.append(self.buf.ptr)
                continue
            p = self.lib.shtns_b200_ipc_open(C.c_char_p(hb))
            if not p:
                capi.check(self.lib)
            self._mapped.append(p)
            ptrs.append(p)
        self.set_row_buffers(ptrs)

    def allocate(self, nfc):
        """This rank's row buffer only (no mapping): [nfc][mmax+1][nrows]."""
        self.release()
        self.buf = RowBuffer(self.lib, (nfc, self.plan.mmax + 1, self.nrows))

    def set_row_buffers(self, ptrs):
        """Device addresses of every rank's row buffer, in rank order."""
        self.ptrs = (C.c_void_p * self.world)(*[C.c_void_p(int(p)) for p in ptrs])
        self.bounds = (C.c_int * (self.world + 1))(*([a for a, _ in self.rows] + [self.plan.nlat]))

    def _spec_ptrs(self, kind, arrs):
        return CudaStages._ptrs(kind, arrs)

    # ---------------- phases (public for callers that order the ranks themselves) ----------------
    def synth_rows(self, *specs, ltr=None):
        """Legendre stage of this rank's orders, rows stored into their owners' buffers."""
        kind = self._kind(len(specs))
        specs = [s.contiguous() for s in specs]
        nf = specs[0].numel() // self.plan.nlm
        self.plan._batch(nf)
        self.plan._stream()
        q = self._spec_ptrs(kind, specs)
        self.lib.shtns_b200_legendre_synth_rows(self.plan._cfg, kind, q[0], q[1], q[2], self.m0, self.m1,
                                                self._ltr(ltr), self.world, self.bounds, self.ptrs)
        capi.check(self.lib)

    def analys_rows(self, n, lead, device, ltr=None):
        """Legendre stage of this rank's orders from the owners' buffers."""
        kind = self._kind(n)
        nf = int(np.prod(lead)) if len(lead) else 1
        outs = [torch.zeros(tuple(lead) + (self.plan.nlm,), dtype=torch.complex128, device=device) for _ in range(n)]
        self.plan._batch(nf)
        self.plan._stream()
        q = self._spec_ptrs(kind, outs)
        self.lib.shtns_b200_legendre_analys_rows(self.plan._cfg, kind, self.world, self.bounds, self.ptrs,
                                                 q[0], q[1], q[2], self.m0, self.m1, self._ltr(ltr))
        capi.check(self.lib)
        return outs

    def own_rows(self, nfc):
        return self.buf.tensor()[:nfc]

    def analys_fourier_rows(self, *blocks, ltr=None):
        """FFT of this rank's blocks into its own row buffer."""
        kind = self._kind(len(blocks))
        blocks = [b.contiguous() for b in blocks]
        bs = self.block_shape()
        nf = blocks[0].numel() // (bs[0] * bs[1])
        self.stages.fourier_analys(kind, blocks, self.own_rows(len(blocks) * nf), self.nrows, self._ltr(ltr), nf)

    # ---------------- whole directions ----------------
    def synth(self, *specs, ltr=None):
        nf = specs[0].numel() // self.plan.nlm
        nfc = len(specs) * nf
        self.prepare(nfc)
        self.barrier()
        self.synth_rows(*specs, ltr=ltr)
        self.barrier()
        outs = self.synth_fourier(self.own_rows(nfc), specs[0].shape[:-1], len(specs), ltr)
        return outs[0] if len(outs) == 1 else tuple(outs)

    def analys(self, *blocks, ltr=None):
        bs = self.block_shape()
        nf = blocks[0].numel() // (bs[0] * bs[1])
        nfc = len(blocks) * nf
        self.prepare(nfc)
        self.barrier()
        self.analys_fourier_rows(*blocks, ltr=ltr)
        self.barrier()
        outs = self.analys_rows(len(blocks), blocks[0].shape[:-2], blocks[0].device, ltr)
        return outs[0] if len(outs) == 1 else tuple(outs)
