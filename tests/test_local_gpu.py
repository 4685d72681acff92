"""Local and partial evaluation on the GPU (points, one latitude, Legendre
arrays, l+-1 operators) against the reference library's own functions
(sht_func.c:453-885, sht_legendre.c:238-440) on the same plans and inputs,
and against the long-double oracle at high degree.  Bar: 1e-12 relative to
the field's largest value (or to the largest array entry)."""
import ctypes as C

import numpy as np
import pytest

from tests.common import rand_spec, relerr

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _ref():
    from oracle import shtns_ref as R
    if not R.available():
        pytest.skip("reference library not built")
    L = R.lib()
    cfg = L.shtns_create.restype
    P, D, I = C.c_void_p, C.c_double, C.c_int
    dp = C.POINTER(C.c_double)

    class Z(C.Structure):
        _fields_ = [("re", C.c_double), ("im", C.c_double)]
    L.SH_to_point_cplx.restype = Z
    L.SH_to_point_cplx.argtypes = [cfg, P, D, D]
    L.SH_to_grad_point.argtypes = [cfg, P, P, D, D, dp, dp, dp]
    L.SHqst_to_point.argtypes = [cfg, P, P, P, D, D, dp, dp, dp]
    L.SH_to_lat.argtypes = [cfg, P, D, P, I, I, I]
    L.SHqst_to_lat.argtypes = [cfg, P, P, P, D, P, P, P, I, I, I]
    L.legendre_sphPlm_deriv_array.restype = I
    L.legendre_sphPlm_deriv_array.argtypes = [cfg, I, I, D, D, P, P]
    L.mul_ct_matrix.argtypes = [cfg, P]
    L.st_dt_matrix.argtypes = [cfg, P]
    L.SH_mul_mx.argtypes = [cfg, P, P, P]
    return R, L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


PLANS = [
    (63, 63, 1, 0),                      # orthonormal
    (127, 40, 2, 0),                     # mres 2, mmax < lmax
    (95, 95, 1, 2),                      # Schmidt
    (80, 80, 1, 1 | 256 * 4 | 256 * 8),  # 4pi, no CS phase, real norm
]
POINTS = [(0.3, 1.1), (-0.7, 5.9), (1.0, 0.4), (-1.0, 2.0), (0.999999, 3.0), (0.0, 0.0), (-0.2, -2.5)]


def _plans(lmax, mmax, mres, norm):
    import shtns_b200
    R, L = _ref()
    nlat = 2 * (lmax + 2)
    nphi = 4 * (mmax * mres + 2)
    ref = R.RefSHT(lmax, mmax, mres, norm, nlat, nphi, flags=R.sht_gauss | R.SHT_THETA_CONTIGUOUS, eps=0.0)
    sh = shtns_b200.sht(lmax, mmax, mres, norm)
    return R, L, ref, sh


@pytest.mark.parametrize("plan", PLANS)
def test_points_match_reference(plan):
    lmax, mmax, mres, norm = plan
    R, L, ref, sh = _plans(*plan)
    q = rand_spec(lmax, mmax, mres, 3)
    s = rand_spec(lmax, mmax, mres, 4, power=1.5, zero_l0=True)
    t = rand_spec(lmax, mmax, mres, 5, power=1.5, zero_l0=True)
    scale = np.abs(ref.synth(q)).max()
    for cost, phi in POINTS:
        a = L.SH_to_point(ref.cfg, _p(q), cost, phi)
        b = sh.SH_to_point(q, cost, phi)
        assert abs(a - b) < TOL * scale, (cost, phi, a, b)
        r3 = [C.c_double() for _ in range(3)]
        L.SHqst_to_point(ref.cfg, _p(q), _p(s), _p(t), cost, phi, *[C.byref(x) for x in r3])
        g3 = sh.SHqst_to_point(q, s, t, cost, phi)
        for x, y in zip(r3, g3):
            assert abs(x.value - y) < TOL * max(scale, 1.0), (cost, phi, x.value, y)
        L.SH_to_grad_point(ref.cfg, _p(q), _p(s), cost, phi, *[C.byref(x) for x in r3])
        g3 = sh.SH_to_grad_point(q, s, cost, phi)
        for x, y in zip(r3, g3):
            assert abs(x.value - y) < TOL * max(scale, 1.0), (cost, phi, x.value, y)
    ref.close()


def test_complex_point_matches_reference():
    R, L, ref, sh = _plans(47, 47, 1, 0)
    rng = np.random.default_rng(9)
    n = 48 * 48
    alm = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) / (1.0 + np.sqrt(np.arange(n)))
    for cost, phi in POINTS:
        z = L.SH_to_point_cplx(ref.cfg, _p(alm), cost, phi)
        w = sh.SH_to_point_cplx(alm, cost, phi)
        assert abs(complex(z.re, z.im) - w) < 1e-12 * np.abs(alm).sum(), (cost, phi)
    ref.close()


@pytest.mark.parametrize("plan", PLANS)
@pytest.mark.parametrize("nphi,ltr,mtr", [(64, None, None), (37, 30, 12), (200, None, None)])
def test_latitude_matches_reference(plan, nphi, ltr, mtr):
    lmax, mmax, mres, norm = plan
    R, L, ref, sh = _plans(*plan)
    q = rand_spec(lmax, mmax, mres, 13)
    s = rand_spec(lmax, mmax, mres, 14, power=1.5, zero_l0=True)
    t = rand_spec(lmax, mmax, mres, 15, power=1.5, zero_l0=True)
    lt = lmax if ltr is None else ltr
    mt = mmax if mtr is None else mtr
    for cost in (0.41, -0.93, 0.0):
        a = np.zeros(nphi)
        L.SH_to_lat(ref.cfg, _p(q), cost, _p(a), nphi, lt, mt)
        b = np.zeros(nphi)
        sh.SH_to_lat(q, cost, b, lt, mt)
        assert relerr(a, b) < TOL
        ra = [np.zeros(nphi) for _ in range(3)]
        L.SHqst_to_lat(ref.cfg, _p(q), _p(s), _p(t), cost, *[_p(x) for x in ra], nphi, lt, mt)
        ga = [np.zeros(nphi) for _ in range(3)]
        sh.SHqst_to_lat(q, s, t, cost, *ga, ltr=lt, mtr=mt)
        for x, y in zip(ra, ga):
            assert relerr(x, y) < TOL
    ref.close()


@pytest.mark.parametrize("plan", PLANS)
def test_legendre_arrays_and_operators_match_reference(plan):
    lmax, mmax, mres, norm = plan
    R, L, ref, sh = _plans(*plan)
    for im in (0, 1, mmax // 2, mmax):
        m = im * mres
        for x in (0.3, -0.95, 0.9999):
            st = np.sqrt((1 - x) * (1 + x))
            a = np.zeros(lmax - m + 1)
            L.legendre_sphPlm_array(ref.cfg, lmax, im, x, a.ctypes.data_as(C.POINTER(C.c_double)))
            b = np.zeros_like(a)
            sh._lib.legendre_sphPlm_array(sh._cfg, lmax, im, x, _p(b))
            assert relerr(a, b) < TOL, (im, x)
            a2, da = np.zeros_like(a), np.zeros_like(a)
            L.legendre_sphPlm_deriv_array(ref.cfg, lmax, im, x, st, _p(a2), _p(da))
            b2, db = np.zeros_like(a), np.zeros_like(a)
            sh._lib.legendre_sphPlm_deriv_array(sh._cfg, lmax, im, x, st, _p(b2), _p(db))
            assert relerr(a2, b2) < TOL and relerr(da, db) < TOL, (im, x)
    q = rand_spec(lmax, mmax, mres, 21)
    for fn in ("mul_ct_matrix", "st_dt_matrix"):
        mx = np.zeros(2 * sh.nlm)
        getattr(L, fn)(ref.cfg, _p(mx))
        mg = getattr(sh, fn)()
        assert relerr(mx, mg) < 1e-15, fn
        r = np.zeros_like(q)
        L.SH_mul_mx(ref.cfg, _p(mx), _p(q), _p(r))
        assert relerr(r, sh.SH_mul_mx(mx, q)) < TOL, fn
    ref.close()


def test_points_high_degree_against_long_double():
    """lmax 1023 at polar, mid and equatorial points: within 1e-12 of the
    long-double sums (the seeds' extended exponent at m near lmax)."""
    import shtns_b200
    from oracle.sht_ld import synth_points
    lmax = 1023
    sh = shtns_b200.sht(lmax)
    q = rand_spec(lmax, lmax, 1, 77)
    xs = np.array([0.9999, 0.5, 0.0, -0.31, -0.99999])
    phis = np.array([0.3, 2.0, 4.4])
    ref = synth_points(q, lmax, xs, phis)            # [nx, nphi]
    got = np.array([[sh.SH_to_point(q, x, ph) for ph in phis] for x in xs])
    assert relerr(ref, got) < TOL


def test_batched_points_equal_single_points():
    import torch
    import shtns_b200
    lmax = 200
    sh = shtns_b200.sht(lmax)
    q = rand_spec(lmax, lmax, 1, 31)
    rng = np.random.default_rng(5)
    ct = np.concatenate([rng.uniform(-1, 1, 500), [1.0, -1.0]])
    ph = rng.uniform(0, 2 * np.pi, ct.size)
    dev = torch.device("cuda:0")
    v = sh.points(torch.from_numpy(q).to(dev), torch.from_numpy(ct).to(dev), torch.from_numpy(ph).to(dev))
    one = np.array([sh.SH_to_point(q, a, b) for a, b in zip(ct[:40], ph[:40])])
    assert np.allclose(v.cpu().numpy()[:40], one, rtol=0, atol=1e-13 * np.abs(one).max())
    # grid check: the points at the plan's own nodes equal the synthesis
    sh.set_grid(302, 432, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_PHI_CONTIGUOUS, polar_opt=0.0)
    grid = sh.synth(q)                               # [nlat, nphi]
    i, j = np.meshgrid(np.arange(0, 302, 7), np.arange(0, 432, 11), indexing="ij")
    pc = torch.from_numpy(sh.cos_theta[i].ravel().copy()).to(dev)
    pp = torch.from_numpy((2 * np.pi * j / 432).ravel()).to(dev)
    v = sh.points(torch.from_numpy(q).to(dev), pc, pp).cpu().numpy()
    assert relerr(grid[i, j].ravel(), v) < TOL
