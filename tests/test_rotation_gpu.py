"""Rotations on the GPU against the reference library's rotation objects,
SH_Zrotate, SH_Yrotate, SH_Yrotate90 and SH_Xrotate90 (sht_func.c:37-385,
1380-2200) on the same inputs and angles, and against point values for the
rotations about y and x (an active rotation R maps the field f to f(R^-1 x)).
Bar: 1e-12 relative to the largest coefficient."""
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
    P, D, I = C.c_void_p, C.c_double, C.c_int
    L.shtns_rotation_create.restype = P
    L.shtns_rotation_create.argtypes = [I, I, I]
    L.shtns_rotation_destroy.argtypes = [P]
    L.shtns_rotation_set_angles_ZYZ.argtypes = [P, D, D, D]
    L.shtns_rotation_set_angles_ZXZ.argtypes = [P, D, D, D]
    L.shtns_rotation_set_angle_axis.argtypes = [P, D, D, D, D]
    L.shtns_rotation_apply_real.argtypes = [P, P, P]
    L.shtns_rotation_apply_cplx.argtypes = [P, P, P]
    L.shtns_rotation_wigner_d_matrix.restype = I
    L.shtns_rotation_wigner_d_matrix.argtypes = [P, I, P]
    L.SH_Zrotate.argtypes = [L.shtns_create.restype, P, D, P]
    L.SH_Yrotate.argtypes = [L.shtns_create.restype, P, D, P]
    L.SH_Yrotate90.argtypes = [L.shtns_create.restype, P, P]
    L.SH_Xrotate90.argtypes = [L.shtns_create.restype, P, P]
    return R, L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


ANGLES = [("zyz", (0.3, 1.1, -0.4)), ("zyz", (0.0, 0.7, 0.0)), ("zyz", (1.0, -0.8, 2.0)), ("zyz", (0.5, 0.0, 0.25)),
          ("zyz", (np.pi / 2, np.pi / 2, -np.pi / 2)), ("zxz", (0.2, 2.5, 0.9)), ("axis", (0.7, 1.0, -2.0, 0.5)),
          ("axis", (1.3, 0.0, 0.0, -1.0))]


def _set(L, r, kind, a):
    fn = {"zyz": "shtns_rotation_set_angles_ZYZ", "zxz": "shtns_rotation_set_angles_ZXZ",
          "axis": "shtns_rotation_set_angle_axis"}[kind]
    getattr(L, fn)(r, *a)


@pytest.mark.parametrize("lmax,mmax,norm", [(40, 40, 0), (127, 127, 0), (64, 30, 0), (50, 50, 256 * 4),
                                            (50, 50, 256 * 8)])
def test_apply_real_matches_reference(lmax, mmax, norm):
    import shtns_b200
    R, L = _ref()
    q = rand_spec(lmax, mmax, 1, 7)
    rr = L.shtns_rotation_create(lmax, mmax, norm)
    rg = shtns_b200.rotation(lmax, mmax, norm)
    for kind, a in ANGLES:
        _set(L, rr, kind, a)
        {"zyz": rg.set_angles_ZYZ, "zxz": rg.set_angles_ZXZ, "axis": rg.set_angle_axis}[kind](*a)
        ref = np.zeros_like(q)
        L.shtns_rotation_apply_real(rr, _p(q), _p(ref))
        got = rg.apply_real(q)
        assert relerr(ref, got) < TOL, (kind, a)
    L.shtns_rotation_destroy(rr)


@pytest.mark.parametrize("lmax", [31, 64])
def test_apply_cplx_and_wigner_match_reference(lmax):
    import shtns_b200
    R, L = _ref()
    rng = np.random.default_rng(4)
    rg = shtns_b200.rotation(lmax)
    n = rg.nlm_cplx
    z = (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    rr = L.shtns_rotation_create(lmax, lmax, 0)
    for kind, a in ANGLES:
        _set(L, rr, kind, a)
        {"zyz": rg.set_angles_ZYZ, "zxz": rg.set_angles_ZXZ, "axis": rg.set_angle_axis}[kind](*a)
        ref = np.zeros_like(z)
        L.shtns_rotation_apply_cplx(rr, _p(z), _p(ref))
        assert relerr(ref, rg.apply_cplx(z)) < TOL, (kind, a)
        if kind == "zyz" and a[1] != 0.0:
            for l in (1, 2, 7, lmax):
                mx = np.zeros((2 * l + 1, 2 * l + 1))
                assert L.shtns_rotation_wigner_d_matrix(rr, l, _p(mx)) == 2 * l + 1
                assert np.abs(mx - rg.wigner_d_matrix(l)).max() < 1e-13, (a, l)
    L.shtns_rotation_destroy(rr)


def test_truncated_complex_rotation_follows_wigner_matrices():
    """mmax < lmax: the rotation of the input padded with zeros above mmax,
    R_l = e^{-i m' gamma} d^l(beta) e^{-i m alpha} Z_l, kept for |m'| <= mmax,
    with the reference's own Wigner matrices.  (The reference's
    shtns_rotation_apply_cplx departs from its matrices for degrees above
    mmax in this case, sht_func.c:1996-2020, so it is not the check here.)"""
    import shtns_b200
    R, L = _ref()
    lmax, mmax = 64, 20
    rng = np.random.default_rng(4)
    rg = shtns_b200.rotation(lmax, mmax)
    n = rg.nlm_cplx
    z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    rr = L.shtns_rotation_create(lmax, lmax, 0)

    def ll(l):
        return l * (l + 1) if l <= mmax else mmax * (2 * l - mmax) + l
    for al, be, ga in ((0.3, 1.1, -0.4), (0.0, 0.7, 0.0), (1.0, 2.9, 1.5)):
        L.shtns_rotation_set_angles_ZYZ(rr, al, be, ga)
        rg.set_angles_ZYZ(al, be, ga)
        want = np.zeros_like(z)
        for l in range(lmax + 1):
            ml = min(l, mmax)
            m = np.arange(-l, l + 1)
            v = np.zeros(2 * l + 1, complex)
            v[l - ml: l + ml + 1] = z[ll(l) - ml: ll(l) + ml + 1]
            mx = np.ones((1, 1))
            if l > 0:
                mx = np.zeros((2 * l + 1, 2 * l + 1))
                L.shtns_rotation_wigner_d_matrix(rr, l, _p(mx))
            out = np.exp(-1j * m * ga) * (mx @ (np.exp(-1j * m * al) * v))
            want[ll(l) - ml: ll(l) + ml + 1] = out[l - ml: l + ml + 1]
        assert relerr(want, rg.apply_cplx(z)) < TOL, (al, be, ga)
    L.shtns_rotation_destroy(rr)


@pytest.mark.parametrize("lmax,mmax,mres", [(60, 60, 1), (90, 30, 3)])
def test_zrotate_matches_reference(lmax, mmax, mres):
    import shtns_b200
    R, L = _ref()
    ref = R.RefSHT(lmax, mmax, mres, 0, 2 * (lmax + 2), 4 * (mmax * mres + 2), flags=R.sht_gauss | 256, eps=0.0)
    sh = shtns_b200.sht(lmax, mmax, mres)
    q = rand_spec(lmax, mmax, mres, 9)
    for alpha in (0.37, -2.0, np.pi / 2):
        a = np.zeros_like(q)
        L.SH_Zrotate(ref.cfg, _p(q), alpha, _p(a))
        assert relerr(a, sh.Zrotate(q, alpha)) < TOL
    ref.close()


def _rmat(axis, ang):
    c, s = np.cos(ang), np.sin(ang)
    if axis == "y":
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])


def test_y_and_x_rotations_are_rotations_of_the_field():
    import shtns_b200
    lmax = 48
    sh = shtns_b200.sht(lmax)
    q = rand_spec(lmax, lmax, 1, 12)
    rng = np.random.default_rng(3)
    pts = [v / np.linalg.norm(v) for v in rng.standard_normal((6, 3))]
    scale = np.abs(q).sum()
    rot = shtns_b200.rotation(lmax)
    for name, axis, ang, out in (("Yrotate", "y", 0.7, sh.Yrotate(q, 0.7)), ("Yrotate90", "y", np.pi / 2, sh.Yrotate90(q)),
                                 ("Xrotate90", "x", np.pi / 2, sh.Xrotate90(q))):
        for v in pts:
            w = _rmat(axis, -ang) @ v
            a = sh.SH_to_point(out, v[2], np.arctan2(v[1], v[0]))
            b = sh.SH_to_point(q, w[2], np.arctan2(w[1], w[0]))
            assert abs(a - b) < 1e-12 * scale, (name, v)
    rot.set_angles_ZYZ(0.0, 0.7, 0.0)
    assert relerr(rot.apply_real(q), sh.Yrotate(q, 0.7)) < 1e-15
    rot.set_angle_axis(np.pi / 2, 1.0, 0.0, 0.0)
    assert relerr(rot.apply_real(q), sh.Xrotate90(q)) < 1e-15


def test_rotation_round_trip_and_norm_at_lmax_1023():
    """A rotation and its inverse give back the input; per-degree energy is
    kept (the rotation is unitary on each degree)."""
    import shtns_b200
    lmax = 1023
    q = rand_spec(lmax, lmax, 1, 44)
    r = shtns_b200.rotation(lmax)
    r.set_angles_ZYZ(0.4, 1.9, -1.2)
    a = r.apply_real(q)
    r.set_angles_ZYZ(1.2, -1.9, -0.4)
    b = r.apply_real(a)
    assert relerr(q, b) < 1e-11
    li = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    mi = np.concatenate([np.full(lmax + 1 - m, m) for m in range(lmax + 1)])
    w = np.where(mi == 0, 1.0, 2.0)
    e0 = np.bincount(li, weights=w * np.abs(q) ** 2)
    e1 = np.bincount(li, weights=w * np.abs(a) ** 2)
    assert np.abs(e1 / e0 - 1).max() < 1e-12


@pytest.mark.parametrize("lmax", [20, 48, 127])
def test_y_and_x_rotations_match_reference(lmax):
    """SH_Yrotate (several angles), SH_Yrotate90 and SH_Xrotate90 against the
    reference's own pseudo-spectral implementation (sht_func.c:101-385)."""
    import shtns_b200
    R, L = _ref()
    ref = R.RefSHT(lmax, lmax, 1, R.sht_orthonormal, 2 * (lmax + 2), 4 * (lmax + 2),
                   flags=R.sht_quick_init | R.SHT_THETA_CONTIGUOUS, eps=0.0)
    sh = shtns_b200.sht(lmax)
    q = rand_spec(lmax, lmax, 1, 21)
    for alpha in (0.7, -1.3, np.pi / 2, 2.9):
        a = np.zeros_like(q)
        L.SH_Yrotate(ref.cfg, _p(q), alpha, _p(a))
        assert relerr(a, sh.Yrotate(q, alpha)) < TOL, alpha
    a = np.zeros_like(q)
    L.SH_Yrotate90(ref.cfg, _p(q), _p(a))
    assert relerr(a, sh.Yrotate90(q)) < TOL
    a = np.zeros_like(q)
    L.SH_Xrotate90(ref.cfg, _p(q), _p(a))
    assert relerr(a, sh.Xrotate90(q)) < TOL
    ref.close()
