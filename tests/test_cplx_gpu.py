"""Complex-valued field transforms (SH_to_spat_cplx, spat_cplx_to_SH and the
sphtor / qst forms) against the reference's own CPU library on the same
plans and inputs, theta- and phi-contiguous layouts, lmax = mmax and
mmax < lmax (C API), plus round trips.  Tolerance 1e-12 relative."""
import ctypes as C

import numpy as np
import pytest

from tests.common import relerr

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P = lambda a: a.ctypes.data_as(C.c_void_p)


def _zspec(rng, lmax, mmax, vector=False):
    out = []
    for l in range(lmax + 1):
        mm = min(l, mmax)
        v = (rng.standard_normal(2 * mm + 1) + 1j * rng.standard_normal(2 * mm + 1)) / (l + 1)
        if vector and l == 0:
            v[:] = 0
        out.append(v)
    return np.concatenate(out)


@pytest.mark.parametrize("mmax,layout", [(47, "theta"), (47, "phi"), (30, "theta")])
def test_cplx_against_reference(mmax, layout):
    import shtns_b200
    from oracle import shtns_ref as R
    if not R.available():
        pytest.skip("reference library not built")
    L, nlat, nphi = 47, 72, 144
    fl = shtns_b200.SHT_THETA_CONTIGUOUS if layout == "theta" else shtns_b200.SHT_PHI_CONTIGUOUS
    sh = shtns_b200.sht(L, mmax)
    sh.set_grid(nlat, nphi, flags=shtns_b200.sht_quick_init | fl, polar_opt=0.0)
    rfl = R.SHT_THETA_CONTIGUOUS if layout == "theta" else R.SHT_PHI_CONTIGUOUS
    ref = R.RefSHT(L, mmax, 1, R.sht_orthonormal, nlat, nphi, flags=R.sht_quick_init | rfl, eps=0.0, nthreads=1)
    RL, lib = R.lib(), sh._lib
    rng = np.random.default_rng(11 + mmax)
    nspat = nlat * nphi
    q = _zspec(rng, L, mmax)
    s = _zspec(rng, L, mmax, True)
    t = _zspec(rng, L, mmax, True)
    for fn_s, fn_a, ins in (("SH_to_spat_cplx", "spat_cplx_to_SH", [q]),
                            ("SHsphtor_to_spat_cplx", "spat_cplx_to_SHsphtor", [s, t]),
                            ("SHqst_to_spat_cplx", "spat_cplx_to_SHqst", [q, s, t])):
        n = len(ins)
        ours = [np.zeros(nspat, dtype=np.complex128) for _ in range(n)]
        theirs = [np.zeros(nspat, dtype=np.complex128) for _ in range(n)]
        getattr(lib, fn_s)(sh._cfg, *[P(a) for a in ins], *[P(o) for o in ours])
        getattr(RL, fn_s)(ref.cfg, *[P(a.copy()) for a in ins], *[P(o) for o in theirs])
        for a, b in zip(ours, theirs):
            assert relerr(b, a) < 1e-12, fn_s
        back = [np.zeros_like(q) for _ in range(n)]
        back_ref = [np.zeros_like(q) for _ in range(n)]
        getattr(lib, fn_a)(sh._cfg, *[P(a) for a in theirs], *[P(o) for o in back])
        getattr(RL, fn_a)(ref.cfg, *[P(a.copy()) for a in theirs], *[P(o) for o in back_ref])
        for a, b, x in zip(back, back_ref, ins):
            assert relerr(b, a) < 1e-12, fn_a
            assert relerr(x, a) < 1e-11, fn_a
    ref.close()


def test_cplx_python_methods():
    import shtns_b200
    sh = shtns_b200.sht(31)
    sh.set_grid(48, 96, flags=shtns_b200.sht_quick_init, polar_opt=0.0)     # phi-contiguous default
    rng = np.random.default_rng(4)
    z = _zspec(rng, 31, 31)
    f = sh.synth_cplx(z)
    assert f.shape == sh.spat_shape and f.dtype == np.complex128
    assert relerr(z, sh.analys_cplx(f)) < 1e-12
    # a real field's complex coefficients: alm[l, -m] = (-1)^m conj alm[l, m]
    q = np.zeros(sh.nlm, dtype=np.complex128)
    q[sh.m > 0] = rng.standard_normal((sh.m > 0).sum()) + 1j * rng.standard_normal((sh.m > 0).sum())
    q[sh.m == 0] = rng.standard_normal((sh.m == 0).sum())
    v = sh.synth(q)
    zc = sh.analys_cplx(v.astype(np.complex128))
    idx = sh.zidx(sh.l, sh.m)
    assert relerr(q, zc[idx]) < 1e-12
    assert np.abs(zc[sh.zidx(sh.l, -sh.m)] - (-1.0) ** sh.m * np.conj(q)).max() < 1e-12
