"""Gauss-Legendre grid generated on the GPU (sht_gauss.cu; the reference's
gauss_nodes, sht_legendre.c:763-811) against the reference library's nodes
and weights and against 40-digit values at sampled nodes.

The GPU refines every node and weight in double-double before rounding, so
they are the correctly rounded values; the reference computes them in long
double and is within a few units in the last place of the nodes (absolute
4e-16) and 1e-9 relative of the weights (its polar weights use P_n' from
before the last Newton step)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _exact(n, z0, digits=40):
    import mpmath
    mpmath.mp.dps = digits
    z = mpmath.mpf(z0)

    def pair(z):
        p1, p2 = z, mpmath.mpf(1)
        for l in range(2, n + 1):
            p1, p2 = ((2 * l - 1) * z * p1 - (l - 1) * p2) / l, p1
        return p1, p2

    for _ in range(3):
        p1, p2 = pair(z)
        z = z - p1 * (1 - z * z) / (n * (p2 - z * p1))
    p1, p2 = pair(z)
    pp = n * (p2 - z * p1)
    return float(z), float(2 * (1 - z * z) / pp ** 2), float(mpmath.sqrt(1 - mpmath.mpf(float(z)) ** 2))


@pytest.mark.parametrize("lmax,nlat", [(127, 192), (511, 768), (1023, 1536), (4095, 6144)])
def test_gpu_gauss_grid_matches_reference_and_exact_values(lmax, nlat):
    import shtns_b200
    from oracle import shtns_ref as R
    sh = shtns_b200.sht(lmax)
    sh.set_grid(nlat, 2 * nlat, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=0.0)
    ct = np.asarray(sh.cos_theta)
    st = np.ctypeslib.as_array(sh._cfg.contents.st, shape=(nlat,)).copy()
    w = sh.gauss_wts()
    n2 = nlat // 2
    assert np.all(np.diff(ct[:n2]) < 0) and np.array_equal(ct[n2:], -ct[:n2][::-1])
    if R.available():
        L = R.lib()
        L.shtns_gauss_wts.argtypes = [L.shtns_create.restype, C.c_void_p]
        lr = min(lmax, 1023)
        ref = R.RefSHT(lr, lr, 1, R.sht_orthonormal, nlat, 2 * nlat,
                       flags=R.sht_quick_init | R.SHT_THETA_CONTIGUOUS, eps=0.0)
        rw = np.zeros(n2)
        L.shtns_gauss_wts(ref.cfg, rw.ctypes.data_as(C.c_void_p))
        assert np.abs(ct - np.asarray(ref.ct[:nlat])).max() < 4e-16
        assert np.abs(w / rw - 1).max() < 1e-9
        ref.close()
    # sampled nodes against 40-digit Newton: equal to the correctly rounded value
    # (1 ulp allowed for values that sit next to a rounding boundary)
    for i in sorted({0, 1, 2, n2 // 7, n2 // 2, n2 - 2, n2 - 1}):
        x, wx, sx = _exact(nlat, ct[i])
        assert abs(ct[i] - x) <= np.spacing(abs(x)), i
        assert abs(w[i] - wx) <= np.spacing(wx), i
        assert abs(st[i] - sx) <= np.spacing(sx), i
