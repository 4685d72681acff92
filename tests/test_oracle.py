"""Pins of the oracle (CPU): the reference library and the NumPy restatement
against the reference's own known-answer test (examples/test_suite.c:96-152),
against each other, and against the committed golden fixtures."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle import sht_np as N
from oracle import shtns_ref as R
from tests.common import rand_spec, relerr

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ref_built = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (make -C oracle)")


def spat_func_test(theta, phi):
    """Analytic field of examples/test_suite.c:90-94 (Y00, Y10, Y20, Y11, Y42)."""
    return (1.0 + 0.01 * np.cos(theta) + 0.1 * (3.0 * np.cos(theta) ** 2 - 1.0)
            + (np.cos(phi) + 0.3 * np.sin(phi)) * np.sin(theta)
            + (np.cos(2 * phi) + 0.1 * np.sin(2 * phi)) * np.sin(theta) ** 2 * (7.0 * np.cos(theta) ** 2 - 1.0) * 3.0 / 8.0)


def kat_expected(idx, nlm):
    """Exact orthonormal coefficients asserted at examples/test_suite.c:124-138."""
    q = np.zeros(nlm, dtype=complex)
    q[0] = np.sqrt(4 * np.pi)
    q[1] = 0.01 * np.sqrt(4 * np.pi / 3)
    q[2] = 0.1 * np.sqrt(16 * np.pi / 5)
    q[idx(1, 1)] = -np.sqrt(2 * np.pi / 3) + 0.3j * np.sqrt(2 * np.pi / 3)
    q[idx(4, 2)] = 0.5 * np.sqrt(2 * np.pi / 5) - 0.05j * np.sqrt(2 * np.pi / 5)
    return q


FTOL = 1e-14   # examples/test_suite.c:14


@ref_built
def test_known_answer_reference_library():
    s = R.RefSHT(7, 3, 1, R.sht_orthonormal, nlat=64, nphi=8, flags=R.sht_quick_init, eps=1e-10)
    theta = np.arccos(s.ct)
    phi = 2 * np.pi * np.arange(8) / 8
    T, P = np.meshgrid(theta, phi)
    d = spat_func_test(T, P)
    q = s.analys(d)
    assert np.abs(q - kat_expected(s.idx, s.nlm)).max() < FTOL
    assert np.abs(s.synth(q) - d).max() < FTOL


def test_known_answer_numpy_restatement():
    s = N.NpSHT(7, 3, 1, N.sht_orthonormal, nlat=64, nphi=8)
    theta = np.arccos(s.ct)
    phi = 2 * np.pi * np.arange(8) / 8
    T, P = np.meshgrid(theta, phi)
    d = spat_func_test(T, P)
    q = s.analys(d)
    assert np.abs(q - kat_expected(s.idx, s.nlm)).max() < FTOL
    assert np.abs(s.synth(q) - d).max() < FTOL


CONFIGS = [
    # lmax, mmax, mres, nlat, nphi, norm, layout, ltr
    (127, 127, 1, 192, 384, N.sht_orthonormal, N.SHT_THETA_CONTIGUOUS, None),
    (31, 10, 2, 48, 64, N.SHT_NO_CS_PHASE, N.SHT_PHI_CONTIGUOUS, None),
    (40, 40, 1, 64, 96, N.sht_fourpi, N.SHT_THETA_CONTIGUOUS, 25),
    (40, 40, 1, 64, 96, N.SHT_REAL_NORM, N.SHT_THETA_CONTIGUOUS, None),
    (64, 60, 1, 96, 128, N.sht_orthonormal, N.SHT_THETA_CONTIGUOUS | N.SHT_SOUTH_POLE_FIRST, None),
]


@ref_built
@pytest.mark.parametrize("cfg", CONFIGS, ids=[f"l{c[0]}m{c[1]}r{c[2]}n{c[5]}f{c[6]}" for c in CONFIGS])
def test_numpy_restatement_matches_reference(cfg):
    lmax, mmax, mres, nlat, nphi, norm, layout, ltr = cfg
    ref = R.RefSHT(lmax, mmax, mres, norm, nlat, nphi, flags=R.sht_quick_init | layout, eps=0.0)
    npo = N.NpSHT(lmax, mmax, mres, norm, nlat, nphi, layout=layout)
    assert np.abs(ref.ct - npo.ct).max() < 4e-16
    q = rand_spec(lmax, mmax, mres, 7)
    s = rand_spec(lmax, mmax, mres, 8, power=1.5, zero_l0=True)
    t = rand_spec(lmax, mmax, mres, 9, power=1.5, zero_l0=True)
    v = ref.synth(q, ltr)
    assert relerr(v, npo.synth(q, ltr)) < 1e-12
    assert relerr(ref.analys(v, ltr), npo.analys(v, ltr)) < 1e-12
    vt, vp = ref.sphtor_synth(s, t, ltr)
    bt, bp = npo.sphtor_synth(s, t, ltr)
    assert relerr(vt, bt) < 1e-12 and relerr(vp, bp) < 1e-12
    rs, rt = ref.sphtor_analys(vt, vp, ltr)
    ns, nt = npo.sphtor_analys(vt, vp, ltr)
    assert relerr(rs, ns) < 1e-12 and relerr(rt, nt) < 1e-12
    ref.close()


def _golden_cases():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def _inputs(meta):
    q = rand_spec(meta["lmax"], meta["mmax"], meta["mres"], meta["seed"], power=1.0)
    s = rand_spec(meta["lmax"], meta["mmax"], meta["mres"], meta["seed"] + 1, power=1.5, zero_l0=True)
    t = rand_spec(meta["lmax"], meta["mmax"], meta["mres"], meta["seed"] + 2, power=1.5, zero_l0=True)
    return q, s, t


@pytest.mark.parametrize("name", sorted(_golden_cases()))
def test_golden_fixtures_match_numpy_restatement(name):
    meta = _golden_cases()[name]
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    if meta["norm"] & 0xFF == N.sht_schmidt:
        pytest.skip("the NumPy restatement covers orthonormal and 4pi normalisations")
    npo = N.NpSHT(meta["lmax"], meta["mmax"], meta["mres"], meta["norm"], meta["nlat"], meta["nphi"],
                  layout=meta["layout"])
    q, s, t = _inputs(meta)
    ltr = meta["ltr"]
    assert np.abs(g["ct"] - npo.ct).max() < 4e-16
    if meta["kind"] == "scalar":
        assert relerr(g["synth_v"], npo.synth(q, ltr)) < 1e-12
        assert relerr(g["analys_q"], npo.analys(g["synth_v"], ltr)) < 1e-12
    elif meta["kind"] == "sphtor":
        vt, vp = npo.sphtor_synth(s, t, ltr)
        assert relerr(g["synth_vt"], vt) < 1e-12 and relerr(g["synth_vp"], vp) < 1e-12
        S, T = npo.sphtor_analys(g["synth_vt"], g["synth_vp"], ltr)
        assert relerr(g["analys_s"], S) < 1e-12 and relerr(g["analys_t"], T) < 1e-12
    else:
        vr, vt, vp = npo.qst_synth(q, s, t, ltr)
        for k, v in (("synth_vr", vr), ("synth_vt", vt), ("synth_vp", vp)):
            assert relerr(g[k], v) < 1e-12, k
        Q, S, T = npo.qst_analys(g["synth_vr"], g["synth_vt"], g["synth_vp"], ltr)
        for k, v in (("analys_q", Q), ("analys_s", S), ("analys_t", T)):
            assert relerr(g[k], v) < 1e-12, k


@ref_built
@pytest.mark.parametrize("name", sorted(_golden_cases()))
def test_golden_fixtures_reproduce_with_reference(name):
    meta = _golden_cases()[name]
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    ref = R.RefSHT(meta["lmax"], meta["mmax"], meta["mres"], meta["norm"], meta["nlat"], meta["nphi"],
                   flags=R.sht_quick_init | meta["layout"], eps=0.0)
    q, s, t = _inputs(meta)
    ltr = meta["ltr"]
    if meta["kind"] == "scalar":
        assert relerr(g["synth_v"], ref.synth(q, ltr)) < 1e-15
    elif meta["kind"] == "sphtor":
        vt, _ = ref.sphtor_synth(s, t, ltr)
        assert relerr(g["synth_vt"], vt) < 1e-15
    else:
        vr, vt, vp = ref.qst_synth(q, s, t, ltr)
        assert relerr(g["synth_vp"], vp) < 1e-15
    ref.close()


@ref_built
def test_round_trip_matches_reference_self_test_bound():
    """SHT_error (sht_init.c:662-738) aborts above 1e-6; the round trip at the
    lmax=127 configuration is at machine precision."""
    ref = R.RefSHT(127, 127, 1, R.sht_orthonormal, 192, 384, flags=R.sht_quick_init | R.SHT_THETA_CONTIGUOUS)
    q = rand_spec(127, 127, 1, 1234)
    assert relerr(q, ref.analys(ref.synth(q))) < 1e-13
    ref.close()


def _fftw(L):
    P, I = C.c_void_p, C.c_int
    IP = C.POINTER(C.c_int)
    L.fftw_plan_many_dft_r2c.restype = P
    L.fftw_plan_many_dft_r2c.argtypes = [I, IP, I, P, IP, I, I, P, IP, I, I, C.c_uint]
    L.fftw_plan_many_dft_c2r.restype = P
    L.fftw_plan_many_dft_c2r.argtypes = [I, IP, I, P, IP, I, I, P, IP, I, I, C.c_uint]
    L.fftw_execute_dft_r2c.argtypes = [P, P, P]
    L.fftw_execute_dft_c2r.argtypes = [P, P, P]
    L.fftw_destroy_plan.argtypes = [P]
    return L


@ref_built
@pytest.mark.parametrize("howmany,nfft", [(33, 48), (9, 16), (127, 384)])
def test_fftw_shim_in_place_strided_r2c_c2r(howmany, nfft):
    """The rotation plan of sht_func.c:86-88: an in-place r2c of `howmany`
    transforms of length nfft, element j of transform t at j*howmany + t
    (istride = ostride = howmany, idist = odist = 1), executed on another
    buffer as at sht_func.c:297; and the c2r of the same layout."""
    L = _fftw(R.lib())
    n = C.c_int(nfft)
    nr, nc = C.c_int(nfft + 2), C.c_int(nfft // 2 + 1)
    buf = np.zeros((nfft + 2) * howmany)
    p = buf.ctypes.data_as(C.c_void_p)
    plan = L.fftw_plan_many_dft_r2c(1, C.byref(n), howmany, p, C.byref(nr), howmany, 1, p, C.byref(nc),
                                    howmany, 1, 64)
    x = np.random.default_rng(5).standard_normal((nfft, howmany))
    work = np.zeros((nfft + 2) * howmany)
    work[:nfft * howmany] = x.ravel()
    w = work.ctypes.data_as(C.c_void_p)
    L.fftw_execute_dft_r2c(plan, w, w)
    got = work.view(np.complex128)[:(nfft // 2 + 1) * howmany].reshape(nfft // 2 + 1, howmany)
    want = np.fft.rfft(x, axis=0)
    assert np.abs(got - want).max() / np.abs(want).max() < 1e-14
    L.fftw_destroy_plan(plan)
    # c2r of the same layout, in place: back to nfft * x
    plan = L.fftw_plan_many_dft_c2r(1, C.byref(n), howmany, p, C.byref(nc), howmany, 1, p, C.byref(nr),
                                    howmany, 1, 64)
    L.fftw_execute_dft_c2r(plan, w, w)
    back = work[:nfft * howmany].reshape(nfft, howmany) / nfft
    assert np.abs(back - x).max() / np.abs(x).max() < 1e-14
    L.fftw_destroy_plan(plan)


def _rmat(axis, ang):
    c, s = np.cos(ang), np.sin(ang)
    if axis == "y":
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])


@ref_built
@pytest.mark.parametrize("lmax", [20, 48])
def test_reference_y_and_x_rotations_are_active_rotations(lmax):
    """SH_Yrotate, SH_Yrotate90 and SH_Xrotate90 (sht_func.c:101-385, the
    pseudo-spectral path through the in-place r2c above) map the field f to
    f(R^-1 x), R the rotation about y (or x) by the angle: checked at points
    with the reference's own SH_to_point."""
    Lb = R.lib()
    cfg = Lb.shtns_create.restype
    P, D = C.c_void_p, C.c_double
    Lb.SH_Yrotate.argtypes = [cfg, P, D, P]
    Lb.SH_Yrotate90.argtypes = [cfg, P, P]
    Lb.SH_Xrotate90.argtypes = [cfg, P, P]
    Lb.SH_to_point.argtypes = [cfg, P, D, D]
    Lb.SH_to_point.restype = D
    ref = R.RefSHT(lmax, lmax, 1, R.sht_orthonormal, 2 * (lmax + 2), 4 * (lmax + 2),
                   flags=R.sht_quick_init | R.SHT_THETA_CONTIGUOUS, eps=0.0)
    q = rand_spec(lmax, lmax, 1, 12)
    ptr = lambda a: a.ctypes.data_as(P)
    scale = np.abs(q).sum()
    pts = [v / np.linalg.norm(v) for v in np.random.default_rng(3).standard_normal((6, 3))]
    for name, axis, ang in (("Yrotate", "y", 0.7), ("Yrotate90", "y", np.pi / 2), ("Xrotate90", "x", np.pi / 2)):
        out = np.zeros_like(q)
        if name == "Yrotate":
            Lb.SH_Yrotate(ref.cfg, ptr(q), ang, ptr(out))
        else:
            getattr(Lb, "SH_" + name)(ref.cfg, ptr(q), ptr(out))
        for v in pts:
            w = _rmat(axis, -ang) @ v
            a = Lb.SH_to_point(ref.cfg, ptr(out), v[2], np.arctan2(v[1], v[0]))
            b = Lb.SH_to_point(ref.cfg, ptr(q), w[2], np.arctan2(w[1], w[0]))
            assert abs(a - b) < 1e-13 * scale, (name, v)
    ref.close()
