"""The reference Python class's in-place transforms and complex-layout
helpers (shtns_numpy.i:319-395, 545-562) give the same results as the
returning forms."""
import numpy as np
import pytest

from tests.common import rand_spec, relerr

pytestmark = pytest.mark.gpu


def test_inplace_transforms_equal_returning_forms():
    import shtns_b200
    sh = shtns_b200.sht(63)
    sh.set_grid(96, 192)
    q, s, t = (rand_spec(63, 63, 1, 40 + i, zero_l0=(i > 0)) for i in range(3))
    v = sh.spat_array()
    sh.SH_to_spat(q, v)
    assert np.array_equal(v, sh.synth(q))
    qb = sh.spec_array()
    sh.spat_to_SH(v, qb)
    assert relerr(q, qb) < 1e-12
    vt, vp = sh.spat_array(), sh.spat_array()
    sh.SHsphtor_to_spat(s, t, vt, vp)
    a, b = sh.synth(s, t)
    assert np.array_equal(vt, a) and np.array_equal(vp, b)
    sh.SHsph_to_spat(s, vt, vp)
    a, b = sh.synth(s, np.zeros_like(t))
    assert np.array_equal(vt, a) and np.array_equal(vp, b)
    sh.SHtor_to_spat(t, vt, vp)
    a, b = sh.synth(np.zeros_like(s), t)
    assert np.array_equal(vt, a) and np.array_equal(vp, b)
    sb, tb = sh.spec_array(), sh.spec_array()
    sh.SHsphtor_to_spat(s, t, vt, vp)
    sh.spat_to_SHsphtor(vt, vp, sb, tb)
    assert relerr(s, sb) < 1e-12 and relerr(t, tb) < 1e-12
    vr = sh.spat_array()
    sh.SHqst_to_spat(q, s, t, vr, vt, vp)
    outs = [sh.spec_array() for _ in range(3)]
    sh.spat_to_SHqst(vr, vt, vp, *outs)
    for x, y in zip((q, s, t), outs):
        assert relerr(x, y) < 1e-12
    with pytest.raises(RuntimeError):
        sh.SH_to_spat(q[:-1], v)


def test_inplace_complex_transforms_and_helpers():
    import shtns_b200
    sh = shtns_b200.sht(31)
    sh.set_grid(48, 64)
    rng = np.random.default_rng(2)
    n = 32 * 32
    alm = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    z = sh.spat_array_cplx()
    sh.SH_to_spat_cplx(alm, z)
    assert np.array_equal(z, sh.synth_cplx(alm))
    back = sh.spec_array_cplx()
    sh.spat_cplx_to_SH(z, back)
    assert relerr(alm, back) < 1e-12
    l, m = sh.zlm(np.arange(n))
    assert all(sh.zidx(int(a), int(b)) == i for i, (a, b) in enumerate(zip(l, m)))
