"""Fixed-order Legendre transforms (the reference's _ml functions: one order,
no FFT) against the reference's own CPU library, same plans and inputs:
every transform family, several orders including 0 and a negative one
(signed m in the vector terms), mres 1 and 2, truncated ltr, and
synthesis / analysis round trips.  Tolerance 1e-12 relative (max norm)."""
import ctypes as C

import numpy as np
import pytest

from tests.common import relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P = lambda a: a.ctypes.data_as(C.c_void_p)


def _plans(L, mres, nlat, nphi):
    import shtns_b200
    from oracle import shtns_ref as R
    if not R.available():
        pytest.skip("reference library not built")
    sh = shtns_b200.sht(L, L // mres, mres)
    sh.set_grid(nlat, nphi, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=0.0)
    ref = R.RefSHT(L, L // mres, mres, R.sht_orthonormal, nlat, nphi,
                   flags=R.sht_quick_init | R.SHT_THETA_CONTIGUOUS, eps=0.0, nthreads=1)
    return sh, ref, R.lib()


def _cvec(rng, n, zero_imag=False):
    v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    if zero_imag:
        v = v.real + 0j
    return v / np.arange(1, n + 1)


@pytest.mark.parametrize("mres", [1, 2])
def test_ml_against_reference(mres):
    L, nlat, nphi = 63, 96, 192
    sh, ref, RL = _plans(L, mres, nlat, nphi)
    lib = sh._lib
    rng = np.random.default_rng(5 + mres)
    orders = [0, 1, 7] if mres == 1 else [0, 3, 10]
    for im in orders + [-orders[1]]:
        m = abs(im) * mres
        nel = L + 1 - m
        for ltr in (L, L - 9):
            q, s, t = (_cvec(rng, nel, m == 0) for _ in range(3))
            # scalar, sphtor, sph, tor, qst synthesis
            cases = [("SH_to_spat_ml", [q], 1), ("SHsphtor_to_spat_ml", [s, t], 2),
                     ("SHsph_to_spat_ml", [s], 2), ("SHtor_to_spat_ml", [t], 2),
                     ("SHqst_to_spat_ml", [q, s, t], 3)]
            for fn, ins, nout in cases:
                ours = [np.zeros(nlat, dtype=np.complex128) for _ in range(nout)]
                theirs = [np.zeros(nlat, dtype=np.complex128) for _ in range(nout)]
                getattr(lib, fn)(sh._cfg, im, *[P(a) for a in ins], *[P(o) for o in ours], ltr)
                getattr(RL, fn)(ref.cfg, C.c_int(im), *[P(a.copy()) for a in ins], *[P(o) for o in theirs], C.c_int(ltr))
                for a, b in zip(ours, theirs):
                    assert relerr(b, a) < 1e-12, (fn, im, ltr)
            # analyses of the reference's fields
            for fn_s, fn_a, nspec in (("SH_to_spat_ml", "spat_to_SH_ml", 1),
                                      ("SHsphtor_to_spat_ml", "spat_to_SHsphtor_ml", 2),
                                      ("SHqst_to_spat_ml", "spat_to_SHqst_ml", 3)):
                ins = [q, s, t][:nspec] if nspec != 2 else [s, t]
                fields = [np.zeros(nlat, dtype=np.complex128) for _ in range(nspec)]
                getattr(RL, fn_s)(ref.cfg, C.c_int(im), *[P(a.copy()) for a in ins], *[P(f) for f in fields], C.c_int(ltr))
                ours = [np.zeros(nel, dtype=np.complex128) for _ in range(nspec)]
                theirs = [np.zeros(nel, dtype=np.complex128) for _ in range(nspec)]
                getattr(lib, fn_a)(sh._cfg, im, *[P(f) for f in fields], *[P(o) for o in ours], ltr)
                getattr(RL, fn_a)(ref.cfg, C.c_int(im), *[P(f.copy()) for f in fields], *[P(o) for o in theirs], C.c_int(ltr))
                kinds = ["q", "s", "t"][:nspec] if nspec != 2 else ["s", "t"]
                for a, b, x, kind in zip(ours, theirs, ins, kinds):
                    assert relerr(b, a) < 1e-12, (fn_a, im, ltr)
                    l = np.arange(nel) + m
                    keep = (l <= ltr) & ((l > 0) | (kind == "q"))   # vector fields have no l = 0 part
                    assert relerr(x[keep], a[keep]) < 1e-12
                    assert np.all(a[l > ltr] == 0)
    ref.close()


def test_ml_python_methods_and_fft_consistency():
    """sht.SH_to_spat_m equals the order-m Fourier coefficient of the full
    synthesis of the same order (v = sum (2 - delta_m0) Re V_m e^{i m phi})."""
    import shtns_b200
    L, nlat, nphi = 47, 72, 144
    sh = shtns_b200.sht(L)
    sh.set_grid(nlat, nphi, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=0.0)
    rng = np.random.default_rng(9)
    for m in (0, 4):
        q = np.zeros(sh.nlm, dtype=np.complex128)
        sel = sh.m == m
        q[sel] = _cvec(rng, int(sel.sum()), m == 0)
        v = sh.synth(q)                                   # [nphi, nlat]
        fm = np.fft.fft(v, axis=0)[m] / nphi
        out = np.zeros(nlat, dtype=np.complex128)
        sh.SH_to_spat_m(np.ascontiguousarray(q[sel]), out, m)
        assert relerr(fm, out) < 1e-13
        back = np.zeros(int(sel.sum()), dtype=np.complex128)
        sh.spat_to_SH_m(out, back, m)
        assert relerr(q[sel], back) < 1e-12
