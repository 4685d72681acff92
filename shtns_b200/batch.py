"""Many scalar fields of uneven lmax, each on its own Gauss grid.

`PlanGroup` wraps the plan-group C API (shtns_b200_group_*): the Legendre
stage of every plan of the group runs as ONE persistent launch whose CTAs take
(plan, order m, tile) work items from a queue sorted by decreasing cost, and
every launch of a group transform goes to one stream.

`UnevenBatch` buckets fields by lmax (one plan per distinct lmax, grid
nlat = 3(lmax+1)/2 rounded up to even, nphi = 2 nlat), keeps the fields of a
bucket in contiguous device buffers, runs synthesis + analysis of all
buckets through a PlanGroup, and can capture that pair of transforms in a
CUDA graph (`capture()` / `replay()`).  It also offers the two slower forms
the group is measured against: one pair of cu_* calls per field
(`pair_per_field`) and one batched pair per bucket (`pair_per_bucket`).

`autotune()` chooses, by timing on the device, the options of each bucket
(latitude pairs per FFT CTA) and of the group (recurrence checkpoint spacing,
work order, CTAs per SM), and caches the choice in a JSON file keyed by
device name and bucket signature.

The reference has no counterpart; its batched interface is shtns_set_batch
(sht_init.c), which handles fields of one lmax only.
"""
import ctypes as C
import json
import os

import numpy as np

from . import capi
from .transforms import sht, sht_quick_init, SHT_THETA_CONTIGUOUS, sht_orthonormal, SHTError

try:
    import torch
except ImportError:
    torch = None


def grid_for(lmax):
    """Gauss grid of a bucket: nlat = 3(lmax+1)/2 rounded up to even, nphi = 2 nlat."""
    nlat = (3 * (lmax + 1) + 1) // 2
    nlat += nlat & 1
    return nlat, 2 * nlat


class PlanGroup:
    """One persistent Legendre launch over several plans (shtns_b200_group_*).

    plans: list of shtns_b200.sht with grids set, on one device.  Transforms
    take per-plan lists of CUDA tensors; a plan with no fields is skipped.
    Launches go to torch's current stream (given to the first plan)."""

    def __init__(self, plans):
        self._lib = capi.load()
        self.plans = list(plans)
        arr = (C.c_void_p * len(self.plans))(*[C.cast(p._cfg, C.c_void_p) for p in self.plans])
        self._g = self._lib.shtns_b200_group_create(len(self.plans), arr)
        if not self._g:
            raise SHTError(self._lib.shtns_b200_last_error().decode())

    def set_option(self, option, value):
        if self._lib.shtns_b200_group_set_option(self._g, int(option), int(value)) != 0:
            raise ValueError("invalid group option %d = %d" % (option, value))

    def _args(self, src, dst):
        n = len(self.plans)
        A = (C.c_void_p * n)(*[x.data_ptr() if x is not None else 0 for x in src])
        B = (C.c_void_p * n)(*[x.data_ptr() if x is not None else 0 for x in dst])
        nf = (C.c_int * n)()
        return A, B, nf

    def synth_into(self, q, v, ltr=None):
        """q[i]: complex128 (nf_i, nlm_i) contiguous; v[i]: float64 (nf_i, *spat_shape_i)."""
        A, B, nf = self._args(q, v)
        for i, (p, x) in enumerate(zip(self.plans, q)):
            nf[i] = 0 if x is None else x.numel() // p.nlm
        self.plans[0]._stream()
        self._lib.shtns_b200_group_synth(self._g, A, B, nf, int(1 << 30 if ltr is None else ltr))
        capi.check(self._lib)

    def analys_into(self, v, q, ltr=None):
        """v[i]: float64 (nf_i, *spat_shape_i); q[i]: complex128 (nf_i, nlm_i)."""
        A, B, nf = self._args(v, q)
        for i, (p, x) in enumerate(zip(self.plans, v)):
            nf[i] = 0 if x is None else x.numel() // p.nspat
        self.plans[0]._stream()
        self._lib.shtns_b200_group_analys(self._g, A, B, nf, int(1 << 30 if ltr is None else ltr))
        capi.check(self._lib)

    @staticmethod
    def _ptrs(lists, n):
        """One C array of device pointers per component list (null entries and
        missing lists give null pointers)."""
        out = []
        for lst in lists:
            if lst is None:
                out.append(None)
            else:
                out.append((C.c_void_p * n)(*[x.data_ptr() if x is not None else 0 for x in lst]))
        return out

    def vector_synth_into(self, spec, spat, ltr=None):
        """Spheroidal/toroidal (spec = (S, T), spat = (Vt, Vp)) or qst
        (spec = (Q, S, T), spat = (Vr, Vt, Vp)) synthesis of every plan: each
        entry a per-plan list of CUDA tensors, complex128 (nf_i, nlm_i) and
        float64 (nf_i, *spat_shape_i)."""
        n = len(self.plans)
        nf = (C.c_int * n)()
        for i, (p, x) in enumerate(zip(self.plans, spec[-1])):
            nf[i] = 0 if x is None else x.numel() // p.nlm
        P = self._ptrs(list(spec) + list(spat), n)
        self.plans[0]._stream()
        lt = int(1 << 30 if ltr is None else ltr)
        if len(spec) == 2:
            self._lib.shtns_b200_group_SHsphtor_to_spat(self._g, *P, nf, lt)
        else:
            self._lib.shtns_b200_group_SHqst_to_spat(self._g, *P, nf, lt)
        capi.check(self._lib)

    def vector_analys_into(self, spat, spec, ltr=None):
        """Analysis counterpart of vector_synth_into (spat = (Vt, Vp) or
        (Vr, Vt, Vp), spec = (S, T) or (Q, S, T))."""
        n = len(self.plans)
        nf = (C.c_int * n)()
        for i, (p, x) in enumerate(zip(self.plans, spat[-1])):
            nf[i] = 0 if x is None else x.numel() // p.nspat
        P = self._ptrs(list(spat) + list(spec), n)
        self.plans[0]._stream()
        lt = int(1 << 30 if ltr is None else ltr)
        if len(spat) == 2:
            self._lib.shtns_b200_group_spat_to_SHsphtor(self._g, *P, nf, lt)
        else:
            self._lib.shtns_b200_group_spat_to_SHqst(self._g, *P, nf, lt)
        capi.check(self._lib)

    def close(self):
        if getattr(self, "_g", None):
            self._lib.shtns_b200_group_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class UnevenBatch:
    """Scalar fields of uneven lmax: one plan and one pair of device buffers
    per distinct lmax (bucket).

    lmaxs: lmax of each field.  Buffers: Q[b] (coefficients, complex128
    (nf_b, nlm_b)), V[b] (grid values, float64 (nf_b, *spat_shape_b)) and
    R[b] (analysis of V[b]).  Field i lives in bucket bucket_of[i], row
    slot_of[i]."""

    def __init__(self, lmaxs, device=None, norm=sht_orthonormal, layout=SHT_THETA_CONTIGUOUS, polar_opt=1.0e-10):
        if torch is None:
            raise RuntimeError("UnevenBatch needs torch")
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.lmaxs = np.asarray(lmaxs, dtype=int)
        if self.lmaxs.ndim != 1 or len(self.lmaxs) == 0:
            raise ValueError("lmaxs must be a non-empty list")
        self.buckets = sorted(set(int(l) for l in self.lmaxs))
        self.bucket_of = np.searchsorted(self.buckets, self.lmaxs)
        self.slot_of = np.zeros(len(self.lmaxs), dtype=int)
        self.count = [0] * len(self.buckets)
        for i, b in enumerate(self.bucket_of):
            self.slot_of[i] = self.count[b]
            self.count[b] += 1
        self.plans = []
        with torch.cuda.device(self.device):
            for l in self.buckets:
                nlat, nphi = grid_for(l)
                sh = sht(l, norm=norm)
                sh.set_grid(nlat, nphi, flags=sht_quick_init | layout, polar_opt=polar_opt)
                self.plans.append(sh)
            self.Q = [torch.zeros((n, sh.nlm), dtype=torch.complex128, device=self.device)
                      for n, sh in zip(self.count, self.plans)]
            self.V = [torch.zeros((n,) + sh.spat_shape, dtype=torch.float64, device=self.device)
                      for n, sh in zip(self.count, self.plans)]
            self.R = [torch.zeros_like(q) for q in self.Q]
            self.group = PlanGroup(self.plans)
        self._graph = None
        self.options = {}

    @property
    def nfields(self):
        return len(self.lmaxs)

    # ---------------- data ----------------
    def set_coefficients(self, coeffs):
        """coeffs: one array (numpy or torch, complex, length nlm of the field's
        lmax) per field, copied into the bucket buffers."""
        for i, c in enumerate(coeffs):
            b, j = self.bucket_of[i], self.slot_of[i]
            t = c if isinstance(c, torch.Tensor) else torch.from_numpy(np.asarray(c, dtype=np.complex128))
            self.Q[b][j].copy_(t.reshape(-1), non_blocking=True)

    def coefficients(self, i):
        return self.Q[self.bucket_of[i]][self.slot_of[i]]

    def grid_values(self, i):
        return self.V[self.bucket_of[i]][self.slot_of[i]]

    def analysed(self, i):
        return self.R[self.bucket_of[i]][self.slot_of[i]]

    # ---------------- transforms ----------------
    def synth(self):
        """Synthesis of every field (Q -> V): one persistent Legendre launch."""
        self.group.synth_into(self.Q, self.V)

    def analys(self):
        """Analysis of every field (V -> R): one persistent Legendre launch."""
        self.group.analys_into(self.V, self.R)

    def pair(self):
        self.synth()
        self.analys()

    def pair_per_bucket(self):
        """Same work as pair(): one batched cu_SH_to_spat + cu_spat_to_SH per bucket."""
        for sh, q, v, r in zip(self.plans, self.Q, self.V, self.R):
            sh.synth_into([q], [v])
            sh.analys_into([v], [r])

    def pair_per_field(self):
        """Same work as pair(): one cu_SH_to_spat + cu_spat_to_SH per field."""
        for sh, q, v, r in zip(self.plans, self.Q, self.V, self.R):
            for j in range(q.shape[0]):
                sh.synth_into([q[j:j + 1]], [v[j:j + 1]])
                sh.analys_into([v[j:j + 1]], [r[j:j + 1]])

    # ---------------- CUDA graph ----------------
    def capture(self, warmup=2):
        """Capture pair() in a CUDA graph (after `warmup` eager pairs, which
        size the work buffers and build the work lists)."""
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self.pair()
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.pair()
        self._graph = g
        return g

    def replay(self):
        if self._graph is None:
            self.capture()
        self._graph.replay()

    def release_graph(self):
        self._graph = None

    # ---------------- options ----------------
    def apply_options(self, opts):
        """opts: {"fft_pairs": [per bucket], "ckseg": c, "order": o, "ctas_per_sm": k}."""
        lib = capi.load()
        for sh, S in zip(self.plans, opts.get("fft_pairs", [])):
            if lib.shtns_b200_set_option(sh._cfg, 1, int(S)) != 0:
                raise ValueError("invalid FFT pairs %r" % S)
        if "ckseg" in opts:
            self.group.set_option(3, opts["ckseg"])
        if "order" in opts:
            self.group.set_option(1, opts["order"])
        if "ctas_per_sm" in opts:
            self.group.set_option(2, opts["ctas_per_sm"])
        self.options = dict(opts)
        self._graph = None


def _time(fn, reps, warm=2):
    for _ in range(warm):
        fn()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def _cache_path(path):
    if path:
        return path
    return os.environ.get("SHTNS_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "shtns_b200", "autotune.json"))


def autotune(batch, reps=3, cache=None, use_cache=True, log=None):
    """Choose the options of an UnevenBatch by timing them on the device.

    Search: for each bucket, latitude pairs per FFT CTA in {1, 2, 4, 8}, timed on
    that bucket's batched transforms; then for the group, checkpoint spacing
    in {8, 16, 32} x work order {cost, natural} x CTAs per SM {2, 3}, timed on
    pair().  The choice is applied, cached (JSON, keyed by device name and the
    (lmax, fields) of each bucket) and returned with the timings."""
    dev = torch.cuda.get_device_name(batch.device)
    key = dev + "|" + ",".join("%dx%d" % (l, n) for l, n in zip(batch.buckets, batch.count))
    path = _cache_path(cache)
    db = {}
    if use_cache and os.path.exists(path):
        try:
            with open(path) as f:
                db = json.load(f)
        except (OSError, ValueError):
            db = {}
    if use_cache and key in db:
        batch.apply_options(db[key]["options"])
        return db[key]
    trials = []
    lib = capi.load()
    pairs = []
    for b, sh in enumerate(batch.plans):
        q, v, r = batch.Q[b], batch.V[b], batch.R[b]

        def run(sh=sh, q=q, v=v, r=r):
            sh.synth_into([q], [v])
            sh.analys_into([v], [r])
        best = None
        for S in (1, 2, 4, 8):
            lib.shtns_b200_set_option(sh._cfg, 1, S)
            t = _time(run, reps)
            trials.append({"bucket": batch.buckets[b], "fft_pairs": S, "ms": t})
            if best is None or t < best[0]:
                best = (t, S)
        pairs.append(best[1])
        lib.shtns_b200_set_option(sh._cfg, 1, best[1])
    best = None
    for seg in (8, 16, 32):
        for order in (0, 1):
            for k in (2, 3):
                opts = {"fft_pairs": pairs, "ckseg": seg, "order": order, "ctas_per_sm": k}
                batch.apply_options(opts)
                t = _time(batch.pair, reps)
                trials.append(dict(opts, ms=t))
                if log:
                    log("autotune %s: %.3f ms" % (opts, t))
                if best is None or t < best[0]:
                    best = (t, opts)
    batch.apply_options(best[1])
    rec = {"options": best[1], "ms": best[0], "trials": trials}
    db[key] = rec
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(db, f, indent=1)
    except OSError:
        pass
    return rec
