"""Benchmark: SH_to_spat + spat_to_SH pairs per second at lmax=511.

Workload (the configuration the headline metric is quoted on): lmax=mmax=511,
mres=1, orthonormal + Condon-Shortley, Gauss grid nlat=768 x nphi=1536,
theta-contiguous, a batch of 64 independent fields (a stack of radial
shells), 3-D vector transforms: one step = SHqst_to_spat then spat_to_SHqst
of all 64 fields.  Coefficients are seeded N(0,1)(l+1)^-p (p = 1 radial,
1.5 spheroidal/toroidal, l=0 zeroed), polar threshold 1e-10 (the SHTns
default) on both arms.  The unit is field-pairs per second (one field-pair =
one 3-component synthesis + analysis of one field).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU (torchrun): fields are independent, every rank transforms its own 64
fields with no collective on the data path (weak scaling); time = max over
ranks of the device-timed region.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LMAX, NLAT, NPHI, NFIELDS, EPS = 511, 768, 1536, 64, 1e-10
E2E_CHUNKS = 16
METRIC = "SH_to_spat+spat_to_SH pairs/s vs lmax; FP64 plain vs batched/split-prec at 1e-11"
UNIT = "field-pairs/s (SHqst_to_spat+spat_to_SHqst, lmax=511, 768x1536)"
WORKLOAD = "lmax511_qst_64fields"


def spectral_inputs(nf, seed):
    from tests.common import rand_spec
    q = rand_spec(LMAX, LMAX, 1, seed, power=1.0, nfields=nf)
    s = rand_spec(LMAX, LMAX, 1, seed + 1, power=1.5, zero_l0=True, nfields=nf)
    t = rand_spec(LMAX, LMAX, 1, seed + 2, power=1.5, zero_l0=True, nfields=nf)
    return q, s, t


# DRAM bytes (read + write) per field of one launch of each Legendre and FFT
# kernel on this workload, from an ncu capture of the 8-field case
# (dram__bytes_read.sum + dram__bytes_write.sum); the traffic grows in
# proportion to the field count.
TRAFFIC_PER_FIELD = {"legendre_synthesis": (98.216960e6 + 92.500992e6) / 8,
                     "legendre_analysis": (153.142784e6 + 34.128384e6) / 8,
                     "fft_synthesis": (152.880640e6 + 178.261760e6) / 8,
                     "fft_analysis": (226.571520e6 + 108.823552e6) / 8}
TRAFFIC_SOURCE = "ncu dram__bytes_read.sum + dram__bytes_write.sum of the 8-field case, scaled by fields"


def legendre_flops(tm, nfields, kind="qst"):
    """Multiply-adds of the even/odd-folded Legendre contraction, x2 flops.
    Per order m, latitude row kept by the polar threshold, field-component and
    Ishioka step k: 4 real FMAs (even/odd x re/im).  Scalar components run
    k < (lmax-m)/2+1, vector components (V, W) k < (lmax+1-m)/2+1."""
    n2 = NLAT // 2
    tot = 0
    for m in range(LMAX + 1):
        rows = n2 - tm[m]
        ks = (LMAX - m) // 2 + 1
        kv = (LMAX + 1 - m) // 2 + 1
        tot += rows * (ks + 2 * kv)          # Q + V + W components
    return 8.0 * tot * nfields


class ClockSampler:
    """nvidia-smi samples of SM clock, power and throttle reasons while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_index):
        self.dev = dev_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.dev)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU side
class quiet_stdout:
    """Route the C library's stdout to /dev/null (the reference's plan set-up
    prints Newton-iteration diagnostics) so that bench.py prints one JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *exc):
        try:
            import ctypes
            ctypes.CDLL(None).fflush(None)
        except OSError:
            pass
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def reference_cpu_rate(target_s=10.0, fields_per_step=None, steps=None, warmup=1, nthreads=None):
    """Field-pairs/s of the reference SHTns CPU library (oracle/_ref: the
    reference's own sources, OpenMP on all host threads, autotuned sht_gauss
    plan) on the same lmax=511 qst workload, one field at a time.  Either runs
    for about target_s seconds or for `steps` steps of `fields_per_step` fields."""
    from oracle import shtns_ref as R
    nthreads = nthreads or os.cpu_count()
    L = R.lib()
    with quiet_stdout():
        ref = R.RefSHT(LMAX, LMAX, 1, R.sht_orthonormal, NLAT, NPHI, flags=R.sht_gauss | R.SHT_THETA_CONTIGUOUS,
                       eps=EPS, nthreads=nthreads)
    nin = NFIELDS
    q, s, t = spectral_inputs(nin, 100)
    sp = [np.zeros((NPHI, NLAT)) for _ in range(3)]
    sq = [np.zeros(ref.nlm, dtype=np.complex128) for _ in range(3)]
    P = lambda a: a.ctypes.data_as(C.c_void_p)

    def pair(f):
        L.SHqst_to_spat(ref.cfg, P(q[f]), P(s[f]), P(t[f]), P(sp[0]), P(sp[1]), P(sp[2]))
        L.spat_to_SHqst(ref.cfg, P(sp[0]), P(sp[1]), P(sp[2]), P(sq[0]), P(sq[1]), P(sq[2]))

    for i in range(max(1, warmup)):
        pair(i % nin)
    n = 0
    t0 = time.perf_counter()
    if steps is None:
        while time.perf_counter() - t0 < target_s or n < 3:
            pair(n % nin)
            n += 1
    else:
        for _ in range(steps):
            for _ in range(fields_per_step):
                pair(n % nin)
                n += 1
    dt = time.perf_counter() - t0
    ref.close()
    return n / dt, n, dt, nthreads


def run_reference(args):
    """--impl reference: the reference's CPU implementation of the path on the
    host cores (rank 0 only under torchrun)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # one step = the GPU arm's step: all NFIELDS field-pairs (the same seeded
    # inputs), one field at a time on all host threads
    fps = NFIELDS
    rate, n, dt, nth = reference_cpu_rate(steps=args.steps, fields_per_step=fps, warmup=args.warmup * fps)
    sample = (f"{args.steps} steps x {fps} field-pairs (the whole {fps}-field step) of the lmax=511 qst workload "
              f"({n} pairs, {dt:.1f} s)")
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "lmax": LMAX, "nlat": NLAT, "nphi": NPHI, "fields_per_step": fps,
                   "polar_eps": EPS, "layout": "theta-contiguous"},
        "impl": "reference",
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": nth, "kind": "reference", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def fp64_gemm_peak(torch, dev):
    """Measured FP64 tensor-core throughput of this GPU: cuBLAS DGEMM 8192^3,
    best of 3 (the FP64 counterpart of the bf16 GEMM figure of
    MEASURED_PEAKS.json, which holds no FP64 number)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def host_array_pair(torch, dev, lib, sh, qn, sn, tn, nf, steps, world, dist):
    """The drop-in host API end to end: SHqst_to_spat then spat_to_SHqst of the
    nf fields with HOST spectral and spatial arrays (page-locked, from
    shtns_malloc, as the reference's users allocate them), wall clock around
    the synchronous calls (max over ranks), beside the link's ceiling for the
    same copies: per call its host->device and device->host bytes moved at
    once on two streams without the transforms."""
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    bufs = []

    def pinned(shape, dtype):
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        ptr = lib.shtns_malloc(n)
        if not ptr:
            raise MemoryError("shtns_malloc")
        bufs.append(ptr)
        return np.frombuffer((C.c_char * n).from_address(ptr), dtype=dtype).reshape(shape)

    try:
        spec = [pinned((nf, sh.nlm), np.complex128) for _ in range(3)]
        for a, src in zip(spec, (qn, sn, tn)):
            a[...] = src
        spat = [pinned((nf,) + sh.spat_shape, np.float64) for _ in range(3)]
        back = [pinned((nf, sh.nlm), np.complex128) for _ in range(3)]
        lib.shtns_set_batch(sh._cfg, nf, sh.nlm, sh.nspat)
        lib.cushtns_set_streams(sh._cfg, C.c_void_p(torch.cuda.current_stream().cuda_stream), None)

        def pair():
            lib.SHqst_to_spat(sh._cfg, *(P(a) for a in spec), *(P(a) for a in spat))
            lib.spat_to_SHqst(sh._cfg, *(P(a) for a in spat), *(P(a) for a in back))

        pair()
        err = max(float(np.abs(a - b).max() / np.abs(a).max()) for a, b in zip(spec, back))
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            pair()
        dt = (time.perf_counter() - t0) / steps
        # the link's ceiling: the same bytes per call, both directions at once
        nspec, nspat = 3 * nf * sh.nlm * 16, 3 * nf * sh.nspat * 8
        d_spec = torch.empty(nspec, dtype=torch.uint8, device=dev)
        d_spat = torch.empty(nspat, dtype=torch.uint8, device=dev)
        h_spec = torch.from_numpy(np.concatenate([a.reshape(-1).view(np.uint8) for a in spec]))
        h_spat = torch.from_numpy(np.concatenate([a.reshape(-1).view(np.uint8) for a in spat])).pin_memory()
        h_spec = h_spec.pin_memory()
        s1, s2 = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)

        def copies():
            with torch.cuda.stream(s1):
                d_spec.copy_(h_spec, non_blocking=True)      # synthesis: spectra in
            with torch.cuda.stream(s2):
                h_spat.copy_(d_spat, non_blocking=True)      # synthesis: grids out
            torch.cuda.synchronize()
            with torch.cuda.stream(s1):
                d_spat.copy_(h_spat, non_blocking=True)      # analysis: grids in
            with torch.cuda.stream(s2):
                h_spec.copy_(d_spec, non_blocking=True)      # analysis: spectra out
            torch.cuda.synchronize()

        copies()
        t0 = time.perf_counter()
        for _ in range(steps):
            copies()
        dl = (time.perf_counter() - t0) / steps
        del d_spec, d_spat, h_spec, h_spat
        if world > 1:
            t = torch.tensor([dt, dl], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt, dl = float(t[0]), float(t[1])
        return {"value": world * nf / dt, "unit": UNIT, "ms_per_step": 1e3 * dt,
                "h2d_bytes_per_step": nspec + nspat, "d2h_bytes_per_step": nspec + nspat,
                "roundtrip_relerr": err,
                "link_ceiling": {"value": world * nf / dl, "ms_per_step": 1e3 * dl,
                                 "note": "the same host<->device bytes per call, both directions at once on two "
                                         "streams, without the transforms, timed in this run"},
                "frac_of_link_ceiling": dl / dt,
                "form": "SHqst_to_spat + spat_to_SHqst with page-locked host arrays (shtns_malloc): the library "
                        "pipelines the fields in chunks over a transfer stream, the compute stream and a second copy "
                        "stream; wall clock around the synchronous calls"}
    finally:
        for ptr in bufs:
            lib.shtns_free(C.c_void_p(ptr))


def cufft_reference_times(torch, dev, spat, nf, reps=5):
    """cuFFT with the reference's theta-contiguous plan (sht_gpu.cu:186-190:
    Z2Z of length nphi over the nlat/2 latitude pairs of one field, one
    execution per field-component, as the reference's cu_* transforms call
    it) over the step's 3 x nf grids, out of place into a buffer of the same
    size.  Milliseconds per direction (all field-components), best of reps.
    cuFFT writes the whole pair spectrum; the library's FFT stages also
    separate the two real spectra of each pair and keep only m <= mmax."""
    from tests import cufft
    st = torch.cuda.current_stream()
    plan = cufft.PairPlan(NPHI, NLAT, st.cuda_stream)
    out = [torch.empty_like(x) for x in spat]
    res = {}
    for name, direction in (("z2z_forward_ms", cufft.CUFFT_FORWARD), ("z2z_inverse_ms", cufft.CUFFT_INVERSE)):
        def run():
            for x, y in zip(spat, out):
                for f in range(nf):
                    plan.exec(x[f].data_ptr(), y[f].data_ptr(), direction)
        run()
        torch.cuda.synchronize()
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run()
            e1.record()
            e1.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        res[name] = best
    plan.destroy()
    del out
    torch.cuda.empty_cache()
    res["plan"] = (f"cufftPlanMany Z2Z n={NPHI}, istride=ostride={NLAT // 2}, idist=odist=1, batch={NLAT // 2}; "
                   f"{3 * nf} executions per direction, out of place")
    return res


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


# ---------------------------------------------------------------- GPU arm
def run_gpu(args):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    import shtns_b200
    from shtns_b200 import capi
    lib = capi.load()
    nf = args.fields
    sh = shtns_b200.sht(LMAX, LMAX, 1)
    sh.set_grid(NLAT, NPHI, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=EPS)
    qn, sn, tn = spectral_inputs(nf, 100 + 7 * rank)
    spec = [torch.from_numpy(a).to(dev) for a in (qn, sn, tn)]
    spat = [torch.empty((nf, NPHI, NLAT), dtype=torch.float64, device=dev) for _ in range(3)]
    back = [torch.empty((nf, sh.nlm), dtype=torch.complex128, device=dev) for _ in range(3)]

    def step():
        sh.synth_into(spec, spat)
        sh.analys_into(spat, back)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    lib.shtns_b200_set_timing(sh._cfg, 1)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    n0 = lib.shtns_b200_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    e1.synchronize()
    launches = lib.shtns_b200_launch_count() - n0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_total = e0.elapsed_time(e1)
    ms_stage = np.zeros(6)
    calls = np.zeros(6, dtype=np.int64)
    lib.shtns_b200_stage_times(sh._cfg, ms_stage.ctypes.data_as(C.c_void_p), calls.ctypes.data_as(C.c_void_p))
    lib.shtns_b200_set_timing(sh._cfg, 0)
    if world > 1:
        t = torch.tensor([ms_total], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    # correctness of what was timed
    rt_err = max(float((a - b).abs().max() / a.abs().max()) for a, b in zip(spec, back))

    # the split-precision form of the same step (INT8 digit table, 7 digits,
    # synthesis and analysis on the INT8 tensor cores), timed the same way
    # after its table is built; errors against the FP64 stages on the same inputs
    split = None
    if not args.no_split:
        spat64 = [x.clone() for x in spat]
        back64 = [x.clone() for x in back]
        sh.set_split(args.split_digits)
        t0b = time.perf_counter()
        step()
        torch.cuda.synchronize()
        build_s = time.perf_counter() - t0b
        for _ in range(args.warmup):
            step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        lib.shtns_b200_set_timing(sh._cfg, 1)
        n0s = lib.shtns_b200_launch_count()
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        e1.synchronize()
        launches_split = lib.shtns_b200_launch_count() - n0s
        ms_split = e0.elapsed_time(e1) / args.steps
        st_s = np.zeros(6)
        ca_s = np.zeros(6, dtype=np.int64)
        lib.shtns_b200_stage_times(sh._cfg, st_s.ctypes.data_as(C.c_void_p), ca_s.ctypes.data_as(C.c_void_p))
        lib.shtns_b200_set_timing(sh._cfg, 0)
        err_syn = max(float((a - b).abs().max() / b.abs().max()) for a, b in zip(spat, spat64))
        sh.analys_into(spat64, back)
        err_ana = max(float((a - b).abs().max() / b.abs().max()) for a, b in zip(back, back64))
        kerr = int(sh.kernel_errors())
        tab = int(lib.shtns_b200_split_table_bytes(sh._cfg))
        sh.set_split(0)
        del spat64, back64
        if world > 1:
            t = torch.tensor([ms_split], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_split = float(t.item())
        per = st_s / np.maximum(ca_s, 1)
        split = {"digits": args.split_digits, "value": world * nf / (ms_split * 1e-3), "ms_per_step": ms_split,
                 "stages_ms": dict(zip(["prologue", "legendre_synthesis", "fft_synthesis", "fft_analysis",
                                        "legendre_analysis", "epilogue"], [float(x) for x in per])),
                 "synth_max_rel_err": err_syn, "analys_max_rel_err": err_ana, "kernel_errors": kerr,
                 "table_bytes": tab, "table_build_s": build_s, "gpu_launches": int(launches_split),
                 "form": "INT8 digit table of the Legendre values (built once per plan), tcgen05 kind::i8 with exact "
                         "INT32 sums, FP64 combine; errors relative to the largest FP64 output"}

    # end to end through the public API: pinned host spectra in, spectra out.
    # The step's fields go in E2E_CHUNKS chunks, each on its own stream with
    # its own plan clone (cushtns_clone), so that the host->device copy of one
    # chunk, the transforms of another and the device->host copy of a third
    # overlap (one copy engine per direction).
    host_in = [torch.from_numpy(a).pin_memory() for a in (qn, sn, tn)]
    host_out = [torch.empty((nf, sh.nlm), dtype=torch.complex128).pin_memory() for _ in range(3)]
    e2e_steps = max(3, min(args.steps, 20))
    nch = max(1, min(args.e2e_chunks, nf))
    bounds = [(c * nf // nch, (c + 1) * nf // nch) for c in range(nch)]
    streams = [torch.cuda.Stream(device=dev) for _ in range(nch)]
    clones = [sh.clone(stream=st.cuda_stream) for st in streams]

    def e2e_step():
        # every chunk stays on its own stream from step to step (its copies and
        # transforms are ordered there), so the next step's host->device
        # copies overlap this step's device->host copies
        for (a, b), st, pl in zip(bounds, streams, clones):
            with torch.cuda.stream(st):
                for d, h in zip(spec, host_in):
                    d[a:b].copy_(h[a:b], non_blocking=True)
                pl.synth_into([x[a:b] for x in spec], [x[a:b] for x in spat])
                pl.analys_into([x[a:b] for x in spat], [x[a:b] for x in back])
                for h, d in zip(host_out, back):
                    h[a:b].copy_(d[a:b], non_blocking=True)

    def fork():
        for st in streams:
            st.wait_stream(torch.cuda.current_stream())

    def join():
        for st in streams:
            torch.cuda.current_stream().wait_stream(st)

    fork()
    for _ in range(2):
        e2e_step()
    join()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    fork()
    for _ in range(e2e_steps):
        e2e_step()
    join()
    f1.record()
    f1.synchronize()
    ms_e2e = f0.elapsed_time(f1) / e2e_steps

    # the link's own ceiling on this machine: the same copies on the same
    # streams and chunks, without the transforms
    def copy_step():
        for (a, b), st in zip(bounds, streams):
            with torch.cuda.stream(st):
                for d, h in zip(spec, host_in):
                    d[a:b].copy_(h[a:b], non_blocking=True)
                for h, d in zip(host_out, back):
                    h[a:b].copy_(d[a:b], non_blocking=True)

    fork()
    copy_step()
    join()
    torch.cuda.synchronize()
    f0.record()
    fork()
    for _ in range(e2e_steps):
        copy_step()
    join()
    f1.record()
    f1.synchronize()
    ms_link = f0.elapsed_time(f1) / e2e_steps
    if world > 1:
        t = torch.tensor([ms_e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    bytes_io = 3 * nf * sh.nlm * 16

    cufft_times = cufft_reference_times(torch, dev, spat, nf) if rank == 0 else None
    host_api = host_array_pair(torch, dev, lib, sh, qn, sn, tn, nf, max(2, min(args.steps, 5)), world, dist)

    if rank == 0:
        ms_step = ms_total / args.steps
        value = world * nf / (ms_step * 1e-3)
        tm = np.zeros(LMAX + 1, dtype=np.int32)
        lib.shtns_b200_polar_rows(sh._cfg, tm.ctypes.data_as(C.c_void_p))
        flops = legendre_flops(tm, nf)
        peak_fp64 = fp64_gemm_peak(torch, dev)
        per_launch = ms_stage / np.maximum(calls, 1)
        share = ms_stage / max(ms_stage.sum(), 1e-30)
        names = ["prologue", "legendre_synthesis", "fft_synthesis", "fft_analysis", "legendre_analysis", "epilogue"]
        dom = 1 + int(np.argmax(ms_stage[1:5]))       # dominant of the Legendre and FFT stages
        peaks = measured_peaks()
        hbm = peaks.get("hbm_gbs", 6650.0)
        fft_bytes = 3 * nf * (NLAT * (LMAX + 1) * 16 + NLAT * NPHI * 8)
        stages = {}
        for i, nm in enumerate(names):
            d = {"ms_per_launch": per_launch[i], "share": share[i]}
            if i in (1, 4):
                d["tflops"] = flops / (per_launch[i] * 1e-3) / 1e12
                d["frac_of_fp64_peak"] = d["tflops"] / peak_fp64
            if i in (2, 3):
                d["gbs"] = fft_bytes / (per_launch[i] * 1e-3) / 1e9
                d["frac_of_hbm"] = d["gbs"] / hbm
            stages[nm] = d
        if dom in (1, 4):
            ach = flops / (per_launch[dom] * 1e-3) / 1e12
            roof = {"kernel": names[dom], "bound": "tensor", "achieved": ach, "peak": peak_fp64,
                    "unit": "TFLOP/s", "frac": ach / peak_fp64, "traffic": TRAFFIC_PER_FIELD[names[dom]] * nf,
                    "traffic_source": TRAFFIC_SOURCE,
                    "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 on the FP64 tensor cores",
                    "work_per_launch": f"{flops:.4e} flop (8 per theta-row x field-component x Ishioka step)"}
        else:
            ach = fft_bytes / (per_launch[dom] * 1e-3) / 1e9
            roof = {"kernel": names[dom], "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                    "frac": ach / hbm, "traffic": TRAFFIC_PER_FIELD[names[dom]] * nf, "traffic_source": TRAFFIC_SOURCE,
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"}
        # the reference's own work count for a transform direction
        # (time_SHT.c:297): W = nlat (4 nlm + 2 (mmax+1) + mmax log2(mmax+1) + 5 nphi log2 nphi)
        # per scalar component; a qst pair counts 2 directions x 3 components
        w1 = NLAT * (4.0 * sh.nlm + 2 * (LMAX + 1) + LMAX * np.log2(LMAX + 1) + 5.0 * NPHI * np.log2(NPHI))
        w_step = 2 * 3 * w1 * nf * world
        roof["reference_work_count"] = {
            "flop_per_step": w_step, "tflops": w_step / (ms_step * 1e-3) / 1e12,
            "frac_of_fp64_peak": w_step / (ms_step * 1e-3) / 1e12 / peak_fp64,
            "note": "whole step (all GPUs) in the reference's operation count (4 flop per degree, order and "
                    "latitude in the Legendre sums); the even/odd folded Ishioka contraction does half of "
                    "those Legendre flops, so this figure is above the kernels' own count"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded N(0,1)(l+1)^-p coefficients)",
            "config": {"workload": WORKLOAD, "lmax": LMAX, "nlat": NLAT, "nphi": NPHI, "fields_per_gpu": nf,
                       "transform": "SHqst_to_spat + spat_to_SHqst", "polar_eps": EPS,
                       "layout": "theta-contiguous", "parallelism": f"fields sharded over {world} GPU(s)",
                       "l2": "no flush: per-step working set %.1f GB > 126 MB L2" %
                             ((3 * nf * sh.nlm * 16 * 2 + 3 * nf * NLAT * NPHI * 8) / 1e9)},
            "roofline": roof,
            "stages": stages,
            "e2e_host_arrays": host_api,
            "split_precision": dict(split, speedup_vs_fp64=split["value"] / value) if split else None,
            "cufft_reference": dict(cufft_times, **{
                "ours_fft_synthesis_ms": float(per_launch[2]), "ours_fft_analysis_ms": float(per_launch[3]),
                "speedup_synthesis": cufft_times["z2z_inverse_ms"] / float(per_launch[2]),
                "speedup_analysis": cufft_times["z2z_forward_ms"] / float(per_launch[3])}) if cufft_times else None,
            "roundtrip_relerr": rt_err,
            "gpu_launches": int(launches),
            "e2e": {"value": world * nf / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": bytes_io,
                    "d2h_bytes_per_step": bytes_io,
                    "form": f"{nch} field chunks on {nch} streams with plan clones: copies overlap transforms "
                            "and the next step's copies",
                    "link_ceiling": {"ms_per_step": ms_link,
                                     "gbs_per_direction": bytes_io / (ms_link * 1e-3) / 1e9,
                                     "value": world * nf / (ms_link * 1e-3),
                                     "note": "the same pinned-host copies on the same streams without the "
                                             "transforms, timed in this run (both directions at once)"}},
            "clocks": clk,
        }
        if world == 1 and not args.no_cpu:
            try:
                rate, n, dt, nth = reference_cpu_rate(target_s=args.cpu_seconds)
                line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": nth, "kind": "reference",
                                        "sample": f"{n} field-pairs of the same workload, one field at a time, "
                                                  f"{dt:.1f} s, reference SHTns 3.5.2 sources (OpenMP, autotuned)"}
            except Exception as e:     # reference library not built on this machine
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(),
                                        "kind": "reference", "sample": f"unavailable: {e}"}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------- uneven lmax
UNEVEN_LMAX = (63, 127, 255, 511, 1023)
UNEVEN_UNIT = "fields/s (SH_to_spat+spat_to_SH of one scalar field on its own grid)"


def uneven_lmaxs(n, seed):
    return np.random.default_rng(seed).choice(UNEVEN_LMAX, size=n)


def uneven_flops(batch):
    """Legendre multiply-adds x2 of one synthesis + one analysis of every field
    (per order m, kept north row and Ishioka step: 4 FMAs per field)."""
    from shtns_b200 import capi
    lib = capi.load()
    tot = 0.0
    for sh, nf in zip(batch.plans, batch.count):
        tm = np.zeros(sh.mmax + 1, dtype=np.int32)
        lib.shtns_b200_polar_rows(sh._cfg, tm.ctypes.data_as(C.c_void_p))
        rows = sh.nlat // 2 - tm
        ks = (sh.lmax - np.arange(sh.mmax + 1)) // 2 + 1
        tot += 8.0 * float((rows * ks).sum()) * nf
    return 2 * tot


def run_uneven(args):
    """256 scalar fields, lmax uniform in {63,...,1023}, each on its own Gauss
    grid nlat=3(lmax+1)/2, nphi=2 nlat: one step = synthesis + analysis of all
    fields.  Forms timed: one cu_* pair per field, one batched pair per lmax
    bucket, the plan group (one persistent Legendre launch per direction)
    eagerly, and the plan group replayed from a CUDA graph (the value)."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    from shtns_b200 import batch as B
    from tests.common import rand_spec
    nf = args.fields if args.fields != NFIELDS else 256
    lm = uneven_lmaxs(nf, 2024)
    ub = B.UnevenBatch(lm, device=dev, polar_opt=EPS)
    for b, (l, n) in enumerate(zip(ub.buckets, ub.count)):
        ub.Q[b].copy_(torch.from_numpy(rand_spec(l, l, 1, 300 + b, power=1.0, nfields=n)))
    tune = B.autotune(ub, use_cache=False)

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    from shtns_b200 import capi
    lib = capi.load()
    ms_field = timed(ub.pair_per_field, max(3, args.steps // 20))
    ms_bucket = timed(ub.pair_per_bucket, args.steps)
    ub.group.set_option(4, 0)          # every launch of the group on one stream
    ms_group1 = timed(ub.pair, args.steps)
    ub.group.set_option(4, 1)          # per-plan launches concurrently on side streams (default)
    ms_group = timed(ub.pair, args.steps)
    ub.capture()
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    ms_graph_persistent = timed(ub.replay, args.steps)
    ub.release_graph()
    # each bucket's own kernels, the buckets concurrently on the group's side
    # streams, captured as parallel branches of one graph
    ub.group.set_option(5, 1)
    ms_group_pp = timed(ub.pair, args.steps)
    ub.capture()
    torch.cuda.synchronize()
    ms_graph_pp = timed(ub.replay, args.steps)
    clk = clocks.stop()
    per_plan = ms_graph_pp < ms_graph_persistent
    ms_graph = min(ms_graph_pp, ms_graph_persistent)
    if not per_plan:
        ub.release_graph()
        ub.group.set_option(5, 0)
        ub.capture()
        torch.cuda.synchronize()
    n0 = lib.shtns_b200_launch_count()
    ub.pair()
    torch.cuda.synchronize()
    launches_pair = lib.shtns_b200_launch_count() - n0
    rt = max(float((q - r).abs().max() / q.abs().max()) for q, r in zip(ub.Q, ub.R))
    flops = uneven_flops(ub)
    peak = fp64_gemm_peak(torch, dev)
    ach = flops / (ms_graph * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": nf / (ms_graph * 1e-3), "unit": UNEVEN_UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_graph, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded N(0,1)/(l+1))",
        "config": {"workload": "uneven_lmax_256fields", "fields": nf,
                   "fields_per_lmax": dict(zip(map(str, ub.buckets), ub.count)),
                   "grids": {str(l): list(B.grid_for(l)) for l in ub.buckets}, "polar_eps": EPS,
                   "layout": "theta-contiguous",
                   "form": "plan group replayed from a CUDA graph (%s)" % (
                       "per-bucket kernels on concurrent graph branches" if per_plan else
                       "one persistent Legendre launch")},
        "forms_fields_per_s": {"per_field_launches": nf / (ms_field * 1e-3),
                               "per_bucket_batched": nf / (ms_bucket * 1e-3),
                               "group_eager_one_stream": nf / (ms_group1 * 1e-3),
                               "group_eager": nf / (ms_group * 1e-3),
                               "group_cuda_graph_persistent_legendre": nf / (ms_graph_persistent * 1e-3),
                               "group_eager_per_bucket_kernels_concurrent": nf / (ms_group_pp * 1e-3),
                               "group_cuda_graph_per_bucket_kernels_concurrent": nf / (ms_graph_pp * 1e-3),
                               "group_cuda_graph": nf / (ms_graph * 1e-3)},
        "speedup_vs_per_field": ms_field / ms_graph,
        "autotune": tune["options"],
        "roofline": {"kernel": "whole step (Legendre flops / step time: lower bound for leg_multi_kernel)",
                     "bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
                     "traffic": None, "peak_source": "measured in this run: cuBLAS DGEMM 8192^3"},
        "roundtrip_relerr": rt,
        "gpu_launches": int(launches_pair),    # per step; the graph replays the same kernels
        "clocks": clk,
    }
    ub.release_graph()
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- high degree
HD_L, HD_NLAT, HD_NPHI, HD_NF = 4095, 6144, 12288, 8
HD_UNIT = "field-pairs/s (SH_to_spat+spat_to_SH, lmax=4095, 6144x12288)"


def run_highdeg(args):
    """lmax=4095 on the 6144 x 12288 Gauss grid, 8 scalar fields: the FP64
    transform pair against the split-precision pair from the precomputed
    INT8 digit table (synthesis and analysis on the INT8 tensor cores, 5, 6
    and 7 digits; 7 is the form within 1e-11), and the on-the-fly FP16
    split synthesis for comparison.  value = pairs/s of the 7-digit table
    form; every form reports its pair, synthesis and Legendre stage times and
    its max / RMS error against the FP64 stages on the same inputs."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    import shtns_b200
    from shtns_b200 import capi
    from tests.common import rand_spec
    lib = capi.load()
    nf = args.fields if args.fields != NFIELDS else HD_NF
    L = args.hd_lmax
    nlat = HD_NLAT if L == HD_L else 3 * (L + 1) // 2 + (3 * (L + 1) // 2) % 2
    nphi = 2 * nlat
    digits = [int(x) for x in args.hd_digits.split(",")]
    sh = shtns_b200.sht(L)
    sh.set_grid(nlat, nphi, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=EPS)
    q = torch.from_numpy(rand_spec(L, L, 1, 400, power=1.0, nfields=nf)).to(dev)
    v = torch.empty((nf,) + sh.spat_shape, dtype=torch.float64, device=dev)
    r = torch.empty_like(q)
    ref = {}

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    def synth():
        sh.synth_into([q], [v])

    def analys():
        sh.analys_into([ref["v64"]], [r])

    def pair():
        sh.synth_into([q], [v])
        sh.analys_into([v], [r])

    def stages(fn):
        lib.shtns_b200_set_timing(sh._cfg, 1)
        fn()
        torch.cuda.synchronize()
        st = np.zeros(6)
        ca = np.zeros(6, dtype=np.int64)
        lib.shtns_b200_stage_times(sh._cfg, st.ctypes.data_as(C.c_void_p), ca.ctypes.data_as(C.c_void_p))
        lib.shtns_b200_set_timing(sh._cfg, 0)
        return st / np.maximum(ca, 1)

    def rel(a, b):
        d, bb = (a - b).abs(), b.abs()
        return float(d.max() / bb.max()), float((d * d).mean().sqrt() / (bb * bb).mean().sqrt())

    steps = max(3, min(args.steps, 10))
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    sh.set_split(0)
    ms_pair = timed(pair, steps)
    ms_syn = timed(synth, steps)
    ref["v64"] = v.clone()
    v64 = ref["v64"]
    ms_ana = timed(analys, steps)
    q64 = r.clone()
    rt = float((q64 - q).abs().max() / q.abs().max())
    st = stages(pair)
    forms = {"fp64": {"pair_ms": ms_pair, "synth_ms": ms_syn, "analys_ms": ms_ana,
                      "legendre_synth_ms": st[1], "legendre_analys_ms": st[4],
                      "pairs_per_s": nf / (ms_pair * 1e-3)}}
    for ns in digits:
        sh.set_split(ns, form=0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        synth()                       # first use builds the digit table
        torch.cuda.synchronize()
        build_s = time.perf_counter() - t0
        ms_s = timed(synth, steps)
        es = rel(v, v64)
        ms_a = timed(analys, steps)
        ea = rel(r, q64)
        ms_p = timed(pair, steps)
        st = stages(pair)
        tab = int(lib.shtns_b200_split_table_bytes(sh._cfg))
        forms["table%d" % ns] = {"pair_ms": ms_p, "synth_ms": ms_s, "analys_ms": ms_a,
                                 "legendre_synth_ms": st[1], "legendre_analys_ms": st[4],
                                 "pairs_per_s": nf / (ms_p * 1e-3), "speedup_vs_fp64": ms_pair / ms_p,
                                 "synth_max_rel_err": es[0], "synth_rms_rel_err": es[1],
                                 "analys_max_rel_err": ea[0], "analys_rms_rel_err": ea[1],
                                 "table_bytes": tab, "table_build_s": build_s,
                                 "kernel_errors": int(sh.kernel_errors())}
    sh.set_split(7, form=1)
    ms_s = timed(synth, steps)
    es = rel(v, v64)
    st = stages(synth)
    forms["fp16_onthefly7"] = {"synth_ms": ms_s, "legendre_synth_ms": st[1], "synth_max_rel_err": es[0],
                               "synth_rms_rel_err": es[1], "kernel_errors": int(sh.kernel_errors())}
    sh.set_split(0)
    clk = clocks.stop()
    tm = np.zeros(L + 1, dtype=np.int32)
    lib.shtns_b200_polar_rows(sh._cfg, tm.ctypes.data_as(C.c_void_p))
    rows = nlat // 2 - tm
    ks = (L - np.arange(L + 1)) // 2 + 1
    flops = 8.0 * float((rows * ks).sum()) * nf
    peak = fp64_gemm_peak(torch, dev)
    hbm = measured_peaks().get("hbm_gbs", 6650.0)
    t7 = forms["table%d" % max(digits)]
    # the table kernels stream the digit table once per launch (plus the
    # digit stacks of the other operand, mostly from L2, and the outputs)
    ach_s = t7["table_bytes"] / (t7["legendre_synth_ms"] * 1e-3) / 1e9
    ach_a = t7["table_bytes"] / (t7["legendre_analys_ms"] * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": nf / (t7["pair_ms"] * 1e-3),
        "unit": "field-pairs/s (SH_to_spat+spat_to_SH, lmax=%d, %dx%d)" % (L, nlat, nphi), "n_gpus": 1, "steps": steps,
        "warmup": args.warmup, "ms_per_step": t7["pair_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8 digits x7, exact int32 sums, f64 combine",
        "data": "synthetic (seeded N(0,1)/(l+1))",
        "config": {"workload": "lmax%d_%dfields" % (L, nf), "lmax": L, "nlat": nlat, "nphi": nphi, "fields": nf,
                   "polar_eps": EPS, "layout": "theta-contiguous",
                   "form": "split precision: %d-digit INT8 table, synthesis + analysis" % max(digits)},
        "split_speedup_vs_fp64": t7["speedup_vs_fp64"],
        "forms": forms,
        "roofline": {"kernel": "ptab_kernel (synthesis / analysis, %d digits)" % max(digits), "bound": "hbm",
                     "achieved": ach_s, "achieved_analysis": ach_a, "peak": hbm, "unit": "GB/s",
                     "frac": ach_s / hbm, "frac_analysis": ach_a / hbm, "traffic": None,
                     "work_per_launch": f"{t7['table_bytes']:.4e} bytes of digit table",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)"},
        "fp64_roofline": {"kernel": "leg_synth_kernel (FP64)", "bound": "tensor",
                          "achieved": flops / (forms["fp64"]["legendre_synth_ms"] * 1e-3) / 1e12, "peak": peak,
                          "unit": "TFLOP/s",
                          "frac": flops / (forms["fp64"]["legendre_synth_ms"] * 1e-3) / 1e12 / peak,
                          "peak_source": "measured in this run: cuBLAS DGEMM 8192^3"},
        "roundtrip_relerr": rt,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_ordersplit(args):
    """One scalar field of lmax=4095 on the 6144 x 12288 grid divided over the
    ranks by order (shtns_b200.ordersplit): each step is a synthesis and an
    analysis, each with one all-to-all of Fourier rows (NCCL between GPUs; a
    copy on one).  The total work is fixed as ranks are added (strong
    scaling); value = field-pairs/s of the whole job, device-timed, max over
    ranks."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    import shtns_b200
    from shtns_b200 import capi
    from shtns_b200.ordersplit import OrderSplit, FusedOrderSplit
    from tests.common import rand_spec
    lib = capi.load()
    nf = args.fields if args.fields != NFIELDS else 1
    sh = shtns_b200.sht(HD_L)
    sh.set_grid(HD_NLAT, HD_NPHI, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=EPS)
    q = torch.from_numpy(rand_spec(HD_L, HD_L, 1, 400, power=1.0, nfields=nf)).to(dev)
    sp = (FusedOrderSplit if args.exchange == "fused" else OrderSplit)(sh, rank=rank, world=world)
    out = {}

    def step():
        v = sp.synth(q)
        out["q"] = sp.analys(v)

    def sync_all():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(max(3, args.warmup)):
        step()
    sync_all()
    steps = max(3, min(args.steps, 20))
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    n0 = lib.shtns_b200_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    e1.synchronize()
    launches = lib.shtns_b200_launch_count() - n0
    sync_all()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / steps
    sl = sp.spec_slice()
    err = float((out["q"][..., sl] - q[..., sl]).abs().max() / q.abs().max())
    # stage times of this rank (one more step, timed per stage)
    lib.shtns_b200_set_timing(sh._cfg, 1)
    step()
    torch.cuda.synchronize()
    st = np.zeros(6)
    ca = np.zeros(6, dtype=np.int64)
    lib.shtns_b200_stage_times(sh._cfg, st.ctypes.data_as(C.c_void_p), ca.ctypes.data_as(C.c_void_p))
    lib.shtns_b200_set_timing(sh._cfg, 0)
    tm = np.zeros(HD_L + 1, dtype=np.int32)
    lib.shtns_b200_polar_rows(sh._cfg, tm.ctypes.data_as(C.c_void_p))
    ims = np.arange(sp.m0, sp.m1 + 1)
    flops = 8.0 * float(((HD_NLAT // 2 - tm[ims]) * ((HD_L - ims) // 2 + 1)).sum()) * nf
    whole_ms = None
    if world == 1:
        # the same field through the whole-field transform, for the cost of the split
        v = torch.empty((nf,) + sh.spat_shape, dtype=torch.float64, device=dev)
        r = torch.empty_like(q)
        for _ in range(2):
            sh.synth_into([q], [v])
            sh.analys_into([v], [r])
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            sh.synth_into([q], [v])
            sh.analys_into([v], [r])
        e1.record()
        e1.synchronize()
        whole_ms = e0.elapsed_time(e1) / steps
    if world > 1:
        t = torch.tensor([ms, err], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, err = float(t[0]), float(t[1])
    if rank == 0:
        peak = fp64_gemm_peak(torch, dev)
        ach = flops / (st[1] * 1e-3) / 1e12 if st[1] > 0 else None
        fourier_bytes = 16.0 * (HD_L + 1) * HD_NLAT * nf
        line = {
            "metric": METRIC, "value": nf / (ms * 1e-3), "unit": HD_UNIT.replace("lmax=4095", "one field, lmax=4095"),
            "n_gpus": world, "steps": steps, "warmup": max(3, args.warmup), "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded N(0,1)/(l+1))",
            "config": {"workload": "lmax4095_1field_ordersplit", "lmax": HD_L, "nlat": HD_NLAT, "nphi": HD_NPHI,
                       "fields": nf, "polar_eps": EPS, "layout": "theta-contiguous",
                       "parallelism": "orders split over %d rank(s), %s" % (world, (
                           "exchange fused into the Legendre kernels (peer row buffers)" if args.exchange == "fused"
                           else "one all-to-all per direction")),
                       "orders_per_rank": [b - a + 1 for a, b in sp.orders],
                       "exchange_bytes_per_step": 2 * fourier_bytes * (world - 1) / max(world, 1),
                       "l2": "no flush: per-step working set > 2 GB > 126 MB L2"},
            "stages_rank0_ms": {"legendre_synthesis": st[1], "fft_synthesis": st[2], "fft_analysis": st[3],
                                "legendre_analysis": st[4], "prologue": st[0], "epilogue": st[5]},
            "roofline": {"kernel": "leg_synth_simt_kernel (FP64 FMA: one field), rank 0's orders", "bound": "fp64",
                         "achieved": ach,
                         "peak": peak, "unit": "TFLOP/s", "frac": ach / peak if ach else None, "traffic": None,
                         "work_per_launch": "8 flop per theta-row x field-component x Ishioka step (the "
                                            "recurrence's 4 more are not counted)",
                         "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 (the FP64 FMA pipe has "
                                        "the same nominal rate on B200)"},
            "roundtrip_relerr": err,
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        if whole_ms is not None:
            line["whole_field_pair_ms"] = whole_ms
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_local(args):
    """Rotations, batched point evaluation and latitude evaluation: the GPU
    forms beside the reference library's own CPU functions on the same inputs
    (host cores, all threads for the rotation).  value = rotations/s of one
    lmax=1023 real field through shtns_rotation_apply_real (host arrays, as the
    reference's API); the other rows are in "rows"."""
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    import shtns_b200
    from shtns_b200 import capi
    from tests.common import rand_spec
    lib = capi.load()
    rows = {}
    clocks = ClockSampler(0)
    clocks.start()

    def wall(fn, reps):
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        return (time.perf_counter() - t0) / reps

    # rotation, lmax 1023, host arrays in and out
    LR = 1023
    q = rand_spec(LR, LR, 1, 5)
    rot = shtns_b200.rotation(LR)
    rot.set_angles_ZYZ(0.4, 1.9, -1.2)
    n0 = lib.shtns_b200_launch_count()
    t_rot = wall(lambda: rot.apply_real(q), 10)
    launches = (lib.shtns_b200_launch_count() - n0) // 11
    rows["rotation_lmax1023"] = {"gpu_ms": t_rot * 1e3, "form": "shtns_rotation_apply_real, host arrays"}
    # batched points, lmax 255, 2^20 points on the device
    LP, NPTS = 255, 1 << 20
    sh = shtns_b200.sht(LP)
    qp = rand_spec(LP, LP, 1, 6)
    rng = np.random.default_rng(1)
    ct = torch.from_numpy(rng.uniform(-1, 1, NPTS)).to(dev)
    ph = torch.from_numpy(rng.uniform(0, 2 * np.pi, NPTS)).to(dev)
    qd = torch.from_numpy(qp).to(dev)
    sh.points(qd, ct, ph)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        sh.points(qd, ct, ph)
    e1.record()
    e1.synchronize()
    t_pts = e0.elapsed_time(e1) / 5 * 1e-3
    rows["points_lmax255"] = {"gpu_points_per_s": NPTS / t_pts, "form": "shtns_b200_SH_to_points, device arrays, 2^20 points"}
    # one latitude, lmax 1023, 2048 longitudes, host arrays
    sl = shtns_b200.sht(LR)
    vl = np.zeros(2048)
    t_lat = wall(lambda: sl.SH_to_lat(q, 0.3, vl), 20)
    rows["latitude_lmax1023"] = {"gpu_ms": t_lat * 1e3, "form": "SH_to_lat, host arrays, nphi 2048"}
    clk = clocks.stop()
    cpu = None
    if not args.no_cpu:
        from oracle import shtns_ref as R
        L = R.lib()
        P = lambda a: a.ctypes.data_as(C.c_void_p)
        L.shtns_rotation_create.restype = C.c_void_p
        L.shtns_rotation_create.argtypes = [C.c_int, C.c_int, C.c_int]
        L.shtns_rotation_set_angles_ZYZ.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.shtns_rotation_apply_real.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.shtns_use_threads(0)
        rr = L.shtns_rotation_create(LR, LR, 0)
        L.shtns_rotation_set_angles_ZYZ(rr, 0.4, 1.9, -1.2)
        out = np.zeros_like(q)
        c_rot = wall(lambda: L.shtns_rotation_apply_real(rr, P(q), P(out)), 3)
        with quiet_stdout():
            ref = R.RefSHT(LP, LP, 1, 0, 384, 768, flags=R.sht_gauss | R.SHT_THETA_CONTIGUOUS, eps=0.0, nthreads=1)
        ctn, phn = ct[:2000].cpu().numpy(), ph[:2000].cpu().numpy()
        t0 = time.perf_counter()
        for a, b in zip(ctn, phn):
            L.SH_to_point(ref.cfg, P(qp), float(a), float(b))
        c_pts = 2000 / (time.perf_counter() - t0)
        ref.close()
        L.SH_to_lat.argtypes = [L.shtns_create.restype, C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_int,
                                C.c_int]
        with quiet_stdout():
            ref = R.RefSHT(LR, LR, 1, 0, 1030, 2060, flags=R.sht_gauss | R.SHT_THETA_CONTIGUOUS, eps=0.0, nthreads=1)
        xs = iter(np.linspace(-0.9, 0.9, 1000))    # a new latitude each call (the reference caches its last one)
        c_lat = wall(lambda: L.SH_to_lat(ref.cfg, P(q), float(next(xs)), P(vl), 2048, LR, LR), 10)
        ref.close()
        rows["rotation_lmax1023"].update({"cpu_ms": c_rot * 1e3, "cpu_threads": os.cpu_count(), "speedup": c_rot / t_rot})
        rows["points_lmax255"].update({"cpu_points_per_s": c_pts, "cpu_threads": 1,
                                       "speedup": rows["points_lmax255"]["gpu_points_per_s"] / c_pts})
        rows["latitude_lmax1023"].update({"cpu_ms": c_lat * 1e3, "cpu_threads": 1, "speedup": c_lat / t_lat})
        cpu = {"value": 1.0 / c_rot, "unit": "rotations/s (lmax=1023, one real field)", "cores": os.cpu_count(),
               "kind": "reference", "sample": "3 rotations of one lmax=1023 field (reference shtns_rotation_apply_real, OpenMP)"}
    line = {
        "metric": "rotations/s, points/s and latitudes/s against the reference CPU functions",
        "value": 1.0 / t_rot, "unit": "rotations/s (lmax=1023, one real field, host arrays)", "n_gpus": 1,
        "steps": 10, "warmup": 1, "ms_per_step": t_rot * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded N(0,1)/(l+1))",
        "config": {"workload": "local_evaluation_and_rotation", "l2": "not flushed (host-array API, wall clock)"},
        "rows": rows, "gpu_launches": int(launches), "cpu_baseline": cpu, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="shtns_b200", choices=["shtns_b200", "reference"])
    ap.add_argument("--fields", type=int, default=NFIELDS)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-split", action="store_true", help="skip the split-precision form of the qst step")
    ap.add_argument("--split-digits", type=int, default=7)
    ap.add_argument("--hd-lmax", type=int, default=HD_L, help="highdeg workload: lmax (grid 3(lmax+1)/2 x 3(lmax+1))")
    ap.add_argument("--hd-digits", default="5,6,7", help="highdeg workload: digit counts of the table form")
    ap.add_argument("--e2e-chunks", type=int, default=E2E_CHUNKS,
                    help="field chunks (streams) of the end-to-end step")
    ap.add_argument("--exchange", default="nccl", choices=["nccl", "fused"],
                    help="ordersplit: NCCL all_to_all_single, or rows stored into peers' buffers by the Legendre kernels")
    ap.add_argument("--workload", default="qst", choices=["qst", "uneven", "highdeg", "ordersplit", "local"],
                    help="qst: lmax=511 vector transforms of 64 fields (default); "
                         "uneven: 256 scalar fields of lmax 63..1023 through a plan group; "
                         "highdeg: lmax=4095, 8 fields, FP64 and split-precision synthesis; "
                         "ordersplit: one lmax=4095 field divided over the ranks by order; "
                         "local: rotations, points and latitudes against the reference functions")
    args = ap.parse_args()
    if args.workload == "uneven" and args.impl != "reference":
        run_uneven(args)
    elif args.workload == "highdeg" and args.impl != "reference":
        run_highdeg(args)
    elif args.workload == "ordersplit" and args.impl != "reference":
        run_ordersplit(args)
    elif args.workload == "local" and args.impl != "reference":
        run_local(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
