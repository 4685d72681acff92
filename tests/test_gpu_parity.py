"""Parity of the CUDA transforms with the reference SHTns 3.5.2 CPU transforms.

Bar (north star): max relative error <= 1e-12 in FP64 (normwise:
max|gpu - ref| / max|ref|), with the reference's kernel choice pinned
(sht_quick_init) and polar threshold 0 unless a test says otherwise.  Inputs
follow the benchmark recipes (tests/common.py).  The references are the
committed golden fixtures (generated from the reference library) and, where
built, the reference library itself in oracle/_ref.
"""
import json
import os

import numpy as np
import pytest

from tests.common import rand_spec, relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-12


def _ref():
    from oracle import shtns_ref as R
    if not R.available():
        pytest.skip("reference library not built")
    return R


def _golden():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def _plan(meta_or_cfg, eps=0.0):
    import shtns_b200
    lmax, mmax, mres, nlat, nphi, norm, layout = meta_or_cfg
    s = shtns_b200.sht(lmax, mmax, mres, norm)
    flags = shtns_b200.sht_quick_init | layout
    if not (layout & shtns_b200.SHT_PHI_CONTIGUOUS):
        flags |= shtns_b200.SHT_THETA_CONTIGUOUS
    s.set_grid(nlat, nphi, flags=flags, polar_opt=eps)
    return s


def _inputs(meta):
    q = rand_spec(meta["lmax"], meta["mmax"], meta["mres"], meta["seed"], power=1.0)
    s = rand_spec(meta["lmax"], meta["mmax"], meta["mres"], meta["seed"] + 1, power=1.5, zero_l0=True)
    t = rand_spec(meta["lmax"], meta["mmax"], meta["mres"], meta["seed"] + 2, power=1.5, zero_l0=True)
    return q, s, t


def _meta_cfg(meta):
    return (meta["lmax"], meta["mmax"], meta["mres"], meta["nlat"], meta["nphi"], meta["norm"], meta["layout"])


@pytest.mark.parametrize("name", sorted(_golden()))
def test_golden_host_api(name):
    """Host-pointer API (SH_to_spat, ... through the Python class)."""
    meta = _golden()[name]
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    sh = _plan(_meta_cfg(meta))
    assert np.abs(sh.cos_theta - g["ct"]).max() < 4e-16
    q, s, t = _inputs(meta)
    ltr = meta["ltr"]
    if meta["kind"] == "scalar":
        assert relerr(g["synth_v"], sh.synth(q, ltr=ltr)) < TOL
        assert relerr(g["analys_q"], sh.analys(g["synth_v"], ltr=ltr)) < TOL
    elif meta["kind"] == "sphtor":
        vt, vp = sh.synth(s, t, ltr=ltr)
        assert relerr(g["synth_vt"], vt) < TOL and relerr(g["synth_vp"], vp) < TOL
        S, T = sh.analys(g["synth_vt"], g["synth_vp"], ltr=ltr)
        assert relerr(g["analys_s"], S) < TOL and relerr(g["analys_t"], T) < TOL
    else:
        vr, vt, vp = sh.synth(q, s, t, ltr=ltr)
        for k, v in (("synth_vr", vr), ("synth_vt", vt), ("synth_vp", vp)):
            assert relerr(g[k], v) < TOL, k
        Q, S, T = sh.analys(g["synth_vr"], g["synth_vt"], g["synth_vp"], ltr=ltr)
        for k, v in (("analys_q", Q), ("analys_s", S), ("analys_t", T)):
            assert relerr(g[k], v) < TOL, k


@pytest.mark.parametrize("name", ["cfg1_scalar", "small_qst", "phi_schmidt_mres2"])
def test_golden_device_api(name):
    """Device-pointer API (cu_* on torch CUDA tensors)."""
    meta = _golden()[name]
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    sh = _plan(_meta_cfg(meta))
    q, s, t = _inputs(meta)
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    ltr = meta["ltr"]
    if meta["kind"] == "scalar":
        v = sh.synth(T(q), ltr=ltr)
        assert relerr(g["synth_v"], v.cpu().numpy()) < TOL
        qa = sh.analys(T(g["synth_v"]), ltr=ltr)
        assert relerr(g["analys_q"], qa.cpu().numpy()) < TOL
    else:
        vr, vt, vp = sh.synth(T(q), T(s), T(t), ltr=ltr)
        for k, v in (("synth_vr", vr), ("synth_vt", vt), ("synth_vp", vp)):
            assert relerr(g[k], v.cpu().numpy()) < TOL, k
        Q, S, Tt = sh.analys(T(g["synth_vr"]), T(g["synth_vt"]), T(g["synth_vp"]), ltr=ltr)
        for k, v in (("analys_q", Q), ("analys_s", S), ("analys_t", Tt)):
            assert relerr(g[k], v.cpu().numpy()) < TOL, k


def test_known_answer_on_gpu():
    """examples/test_suite.c:96-152 through the GPU path (ftol 1e-14)."""
    from tests.test_oracle import spat_func_test, kat_expected
    import shtns_b200
    sh = shtns_b200.sht(7, 3, 1)
    sh.set_grid(64, 8, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=1e-10)
    theta = np.arccos(sh.cos_theta)
    phi = 2 * np.pi * np.arange(8) / 8
    Tg, Pg = np.meshgrid(theta, phi)
    d = spat_func_test(Tg, Pg)
    q = sh.analys(d)
    assert np.abs(q - kat_expected(sh.idx, sh.nlm)).max() < 1e-14
    assert np.abs(sh.synth(q) - d).max() < 1e-14


@pytest.mark.parametrize("kind", ["scalar", "sphtor", "qst"])
def test_batch_equals_single_fields(kind):
    cfg = (63, 63, 1, 96, 192, 0, 256)
    sh = _plan(cfg)
    nf = 5
    q = rand_spec(63, 63, 1, 11, nfields=nf)
    s = rand_spec(63, 63, 1, 12, power=1.5, zero_l0=True, nfields=nf)
    t = rand_spec(63, 63, 1, 13, power=1.5, zero_l0=True, nfields=nf)
    args = {"scalar": (q,), "sphtor": (s, t), "qst": (q, s, t)}[kind]
    out = sh.synth(*args)
    out = out if isinstance(out, tuple) else (out,)
    for f in range(nf):
        one = sh.synth(*(a[f] for a in args))
        one = one if isinstance(one, tuple) else (one,)
        for a, b in zip(out, one):
            assert np.array_equal(a[f], b)
    back = sh.analys(*out)
    back = back if isinstance(back, tuple) else (back,)
    for a, b in zip(args, back):
        assert relerr(a, b) < TOL


@pytest.mark.parametrize("cfg", [
    (127, 127, 1, 192, 384, 0, 256),
    (255, 255, 1, 384, 768, 0, 256),
    (100, 70, 1, 160, 150, 0, 512),            # nphi = 2*3*5*5, phi-contiguous
    (60, 20, 3, 90, 140, 0, 256),              # mres = 3, nphi with radix 7
])
def test_against_reference_library(cfg):
    R = _ref()
    lmax, mmax, mres, nlat, nphi, norm, layout = cfg
    ref = R.RefSHT(lmax, mmax, mres, norm, nlat, nphi, flags=R.sht_quick_init | layout, eps=0.0, nthreads=8)
    sh = _plan(cfg)
    q = rand_spec(lmax, mmax, mres, 21)
    s = rand_spec(lmax, mmax, mres, 22, power=1.5, zero_l0=True)
    t = rand_spec(lmax, mmax, mres, 23, power=1.5, zero_l0=True)
    vr, vt, vp = ref.qst_synth(q, s, t)
    gr, gt, gp = sh.synth(q, s, t)
    assert relerr(vr, gr) < TOL and relerr(vt, gt) < TOL and relerr(vp, gp) < TOL
    Q, S, T = ref.qst_analys(vr, vt, vp)
    gQ, gS, gT = sh.analys(vr, vt, vp)
    assert relerr(Q, gQ) < TOL and relerr(S, gS) < TOL and relerr(T, gT) < TOL
    # truncated forms
    ltr = lmax // 2
    assert relerr(ref.synth(q, ltr), sh.synth(q, ltr=ltr)) < TOL
    assert relerr(ref.analys(vr, ltr), sh.analys(vr, ltr=ltr)) < TOL
    a = ref.sphtor_analys(vt, vp, ltr)
    b = sh.analys(vt, vp, ltr=ltr)
    assert relerr(a[0], b[0]) < TOL and relerr(a[1], b[1]) < TOL
    ref.close()


def test_polar_threshold_matches_reference_within_eps():
    """With the polar threshold on (eps=1e-10, the reference default), both
    sides drop rows whose Legendre values stay below eps; the reference rounds
    the start row down to its SIMD width, so they agree to O(eps)."""
    R = _ref()
    cfg = (255, 255, 1, 384, 768, 0, 256)
    ref = R.RefSHT(255, 255, 1, 0, 384, 768, flags=R.sht_quick_init | 256, eps=1e-10, nthreads=8)
    sh = _plan(cfg, eps=1e-10)
    q = rand_spec(255, 255, 1, 31)
    v = ref.synth(q)
    assert relerr(v, sh.synth(q)) < 1e-9
    assert relerr(ref.analys(v), sh.analys(v)) < 1e-9
    ref.close()


def test_lmax511_vector_batch_against_reference():
    """Configuration-2 sizes (lmax=511, 768 x 1536) on a small batch."""
    R = _ref()
    ref = R.RefSHT(511, 511, 1, 0, 768, 1536, flags=R.sht_quick_init | 256, eps=0.0, nthreads=16)
    sh = _plan((511, 511, 1, 768, 1536, 0, 256))
    nf = 2
    q = rand_spec(511, 511, 1, 41, nfields=nf)
    s = rand_spec(511, 511, 1, 42, power=1.5, zero_l0=True, nfields=nf)
    t = rand_spec(511, 511, 1, 43, power=1.5, zero_l0=True, nfields=nf)
    gr, gt, gp = sh.synth(q, s, t)
    gQ, gS, gT = sh.analys(gr, gt, gp)
    for f in range(nf):
        vr, vt, vp = ref.qst_synth(q[f], s[f], t[f])
        assert relerr(vr, gr[f]) < TOL and relerr(vt, gt[f]) < TOL and relerr(vp, gp[f]) < TOL
        Q, S, T = ref.qst_analys(vr, vt, vp)
        assert relerr(Q, gQ[f]) < TOL and relerr(S, gS[f]) < TOL and relerr(T, gT[f]) < TOL
    ref.close()


def test_lmax511_64_fields_round_trip():
    """Full configuration-2 batch: 64 qst fields; analysis(synthesis(x)) = x."""
    import shtns_b200
    sh = _plan((511, 511, 1, 768, 1536, 0, 256))
    dev = torch.device("cuda:0")
    nf = 64
    q = torch.from_numpy(rand_spec(511, 511, 1, 51, nfields=nf)).to(dev)
    s = torch.from_numpy(rand_spec(511, 511, 1, 52, power=1.5, zero_l0=True, nfields=nf)).to(dev)
    t = torch.from_numpy(rand_spec(511, 511, 1, 53, power=1.5, zero_l0=True, nfields=nf)).to(dev)
    vr, vt, vp = sh.synth(q, s, t)
    Q, S, T = sh.analys(vr, vt, vp)
    for a, b in ((q, Q), (s, S), (t, T)):
        assert relerr(a.cpu().numpy(), b.cpu().numpy()) < TOL
    assert shtns_b200.capi.load().shtns_b200_status() == 0


def test_float_device_transforms():
    """cu_SH_to_spat_float / cu_spat_to_SH_float (FP32 arrays, FP64 inside)."""
    import ctypes as C
    from shtns_b200 import capi
    lib = capi.load()
    sh = _plan((127, 127, 1, 192, 384, 0, 256))
    dev = torch.device("cuda:0")
    q64 = torch.from_numpy(rand_spec(127, 127, 1, 61)).to(dev)
    v64 = sh.synth(q64)
    q32 = q64.to(torch.complex64)
    v32 = torch.empty(sh.spat_shape, dtype=torch.float32, device=dev)
    sh._batch(1)
    sh._stream()
    lib.cu_SH_to_spat_float(sh._cfg, C.c_void_p(q32.data_ptr()), C.c_void_p(v32.data_ptr()), 127)
    back = torch.empty(sh.nlm, dtype=torch.complex64, device=dev)
    lib.cu_spat_to_SH_float(sh._cfg, C.c_void_p(v32.data_ptr()), C.c_void_p(back.data_ptr()), 127)
    torch.cuda.synchronize()
    assert lib.shtns_b200_status() == 0
    assert relerr(v64.cpu().numpy(), v32.double().cpu().numpy()) < 1e-6
    assert relerr(q64.cpu().numpy(), back.to(torch.complex128).cpu().numpy()) < 1e-6


def test_legendre_tile_shapes_agree():
    """Option 5 (Legendre tile shape: 32x128, 64x64, 128x32): the same sums in
    the same order, so synthesis and analysis agree bit for bit."""
    import shtns_b200
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    sh = shtns_b200.sht(255)
    sh.set_grid(384, 768, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=1e-10)
    q = torch.from_numpy(rand_spec(255, 255, 1, 21, nfields=12)).to(dev)
    outs = []
    for wm in (2, 4, 1, 0):
        assert lib.shtns_b200_set_option(sh._cfg, 5, wm) == 0
        v = sh.synth(q)
        outs.append((v, sh.analys(v)))
    assert lib.shtns_b200_set_option(sh._cfg, 5, 3) == -1
    for v, r in outs[1:]:
        assert torch.equal(v, outs[0][0]) and torch.equal(r, outs[0][1])


@pytest.mark.parametrize("case", ["scalar1", "scalar2", "scalar3", "scalar4", "qst_mres2", "sphtor_south_robert",
                                  "scalar1_l2047"])
def test_simt_legendre_matches_tensor_tiles(case):
    """Option 5 = 8 (SIMT kernels, 1-4 field-components) against the tensor-core
    tiles (option 5 = 2) on the same plan: synthesis, analysis and the scalar
    adjoints agree to rounding (different summation order)."""
    import ctypes as C
    import shtns_b200
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    lmax, mmax, mres, nlat, nphi, nf, kind = 255, 255, 1, 384, 768, 1, 0
    flags = shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS
    robert = False
    if case.startswith("scalar") and case[6:].isdigit():
        nf = int(case[6:])
    elif case == "qst_mres2":
        lmax, mmax, mres, nlat, nphi, nf, kind = 191, 60, 2, 288, 384, 1, 2
        flags = shtns_b200.sht_quick_init | shtns_b200.SHT_PHI_CONTIGUOUS
    elif case == "sphtor_south_robert":
        nf, kind, robert = 2, 1, True
        flags |= shtns_b200.SHT_SOUTH_POLE_FIRST
    elif case == "scalar1_l2047":
        lmax, mmax, nlat, nphi = 2047, 2047, 3072, 6144
    sh = shtns_b200.sht(lmax, mmax, mres)
    sh.set_grid(nlat, nphi, flags=flags, polar_opt=1e-10)
    if robert:
        sh.robert_form(1)
    ncomp = {0: 1, 1: 2, 2: 3}[kind]
    specs = [torch.from_numpy(rand_spec(lmax, mmax, mres, 40 + i, nfields=nf, zero_l0=(kind > 0))).to(dev)
             for i in range(ncomp)]
    res = {}
    for opt in (2, 8):
        assert lib.shtns_b200_set_option(sh._cfg, 5, opt) == 0
        v = sh.synth(*specs)
        v = list(v) if isinstance(v, tuple) else [v]
        back = sh.analys(*v)
        back = list(back) if isinstance(back, tuple) else [back]
        res[opt] = (v, back)
        if kind == 0 and nf == 1:
            g = torch.empty_like(specs[0])
            lib.cu_SH_to_spat_adjoint(sh._cfg, C.c_void_p(v[0].data_ptr()), C.c_void_p(g.data_ptr()), lmax)
            h = torch.empty_like(v[0])
            lib.cu_spat_to_SH_adjoint(sh._cfg, C.c_void_p(specs[0].data_ptr()), C.c_void_p(h.data_ptr()), lmax)
            torch.cuda.synchronize()
            res[opt] += (g, h)
    for a, b in zip(res[2][0] + res[2][1], res[8][0] + res[8][1]):
        assert relerr(a.cpu().numpy(), b.cpu().numpy()) < 1e-13
    if len(res[2]) > 2:
        for a, b in zip(res[2][2:], res[8][2:]):
            assert relerr(a.cpu().numpy(), b.cpu().numpy()) < 1e-13
    for a, b in zip(specs, res[8][1]):
        assert relerr(a.cpu().numpy(), b.cpu().numpy()) < 1e-11


@pytest.mark.parametrize("case", ["l511_theta_qst", "l1023_theta", "l255_phi_qst", "l100_ragged", "l63_theta",
                                  "l511_nlat770_ltr"])
def test_prefetched_fft_matches_direct(case):
    """Option 3 (FFT kernels): the automatic choice, persistent CTAs that fetch
    their next latitude tile with tensor copies (option 6 reports 2) and on
    theta-contiguous grids store whole synthesis tiles with tensor stores
    (phi-contiguous analysis keeps the direct kernel), computes the
    same passes as the same kernels with per-thread stores (option 3 = 3) and
    as the direct-load fused kernels (option 3 = 2): results agree bit for
    bit, and with the generic mixed-radix kernels to rounding."""
    import shtns_b200
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    L, nlat, nphi, nf, ncomp, phi, ltr = {
        "l511_theta_qst": (511, 768, 1536, 8, 3, False, None),
        "l1023_theta": (1023, 1536, 3072, 2, 1, False, None),
        "l255_phi_qst": (255, 384, 768, 4, 3, True, None),
        "l100_ragged": (100, 150, 384, 3, 1, False, None),
        "l63_theta": (63, 96, 192, 16, 1, False, None),
        "l511_nlat770_ltr": (511, 770, 1536, 2, 3, False, 300),
    }[case]
    sh = shtns_b200.sht(L)
    layout = shtns_b200.SHT_PHI_CONTIGUOUS if phi else shtns_b200.SHT_THETA_CONTIGUOUS
    sh.set_grid(nlat, nphi, flags=shtns_b200.sht_quick_init | layout, polar_opt=1e-10)
    specs = [torch.from_numpy(rand_spec(L, L, 1, 60 + i, nfields=nf, zero_l0=(ncomp > 1 and i > 0))).to(dev)
             for i in range(ncomp)]
    kw = {} if ltr is None else {"ltr": ltr}
    res = {}
    for opt in (0, 3, 2, 1):
        assert lib.shtns_b200_set_option(sh._cfg, 3, opt) == 0
        spat = [torch.empty((nf,) + sh.spat_shape, dtype=torch.float64, device=dev) for _ in range(ncomp)]
        sh.synth_into(specs, spat, **kw)
        path_s = lib.shtns_b200_get_option(sh._cfg, 6)
        back = [torch.empty_like(x) for x in specs]
        sh.analys_into(spat, back, **kw)
        path_a = lib.shtns_b200_get_option(sh._cfg, 6)
        torch.cuda.synchronize()
        res[opt] = (spat, back, path_s, path_a)
    assert lib.shtns_b200_kernel_errors(sh._cfg) == 0
    ana = 1 if phi else 2             # phi-contiguous analysis keeps the direct kernel
    assert res[0][2:] == (2, ana) and res[3][2:] == (2, ana) and res[2][2:] == (1, 1) and res[1][2:] == (0, 0)
    for o in (3, 2):
        for a, b in zip(res[0][0] + res[0][1], res[o][0] + res[o][1]):
            assert torch.equal(a, b)
    for a, b in zip(res[0][0] + res[0][1], res[1][0] + res[1][1]):
        assert float((a - b).abs().max()) <= 1e-13 * float(b.abs().max())
    assert lib.shtns_b200_set_option(sh._cfg, 3, 4) == -1


def test_prefetched_fft_wait_limit_reports_and_recovers():
    """The prefetching FFT kernels wait on an mbarrier for their tensor copies
    with a time limit.  Option 7 makes them expect 16 bytes more than the
    copies bring, so the wait gives up after about a second: the kernel sets
    the error flag that shtns_b200_kernel_errors reads (and clears) and
    returns without storing.  The context stays usable: the next transforms
    on the same plan are correct."""
    import shtns_b200
    from shtns_b200 import capi
    lib = capi.load()
    dev = torch.device("cuda:0")
    L = 63
    sh = shtns_b200.sht(L)
    sh.set_grid(96, 192, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=0.0)
    q = torch.from_numpy(rand_spec(L, L, 1, 71, nfields=2)).to(dev)
    v = torch.empty((2,) + sh.spat_shape, dtype=torch.float64, device=dev)
    assert lib.shtns_b200_kernel_errors(sh._cfg) == 0
    assert lib.shtns_b200_set_option(sh._cfg, 7, 8) == -1          # not a multiple of 16
    assert lib.shtns_b200_set_option(sh._cfg, 7, 16) == 0
    sh.synth_into([q], [v])
    assert lib.shtns_b200_get_option(sh._cfg, 6) == 2             # the prefetching kernel ran
    assert lib.shtns_b200_kernel_errors(sh._cfg) == 1
    assert lib.shtns_b200_kernel_errors(sh._cfg) == 0             # cleared by the read
    assert lib.shtns_b200_set_option(sh._cfg, 7, 0) == 0
    v = sh.synth(q)
    back = sh.analys(v)
    assert lib.shtns_b200_kernel_errors(sh._cfg) == 0
    assert relerr(q.cpu().numpy(), back.cpu().numpy()) < 1e-12
