"""High-degree FP64 transforms: lmax=mmax=4095, Gauss 6144 x 12288.

Above degree ~1800 the recurrence seed sin^m(theta) leaves the double range
at latitudes where P_l^m later grows to O(1); the checkpoint kernel carries an
extended exponent there.  Checks:
  * synthesis against a long-double evaluation (oracle.sht_ld) at polar,
    mid-latitude and equatorial rows, for all orders and for orders m >= 2000
    only (the range where the seed underflows), to 1e-11 of the field's
    maximum;
  * synthesis and analysis against the reference's CPU library (built from its
    sources, with its own extended-exponent scaling), no polar threshold, to
    1e-11 relative (max norm);
  * the 12288-point fused FFT chain through a batched round trip.
"""
import numpy as np
import pytest

from tests.common import rand_spec, relerr, lm_arrays

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

LMAX, NLAT, NPHI = 4095, 6144, 12288


@pytest.fixture(scope="module")
def plan():
    import shtns_b200
    sh = shtns_b200.sht(LMAX)
    sh.set_grid(NLAT, NPHI, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=0.0)
    return sh


@pytest.fixture(scope="module")
def ref():
    from oracle import shtns_ref as R
    if not R.available():
        pytest.skip("reference library not built")
    r = R.RefSHT(LMAX, LMAX, 1, R.sht_orthonormal, NLAT, NPHI,
                 flags=R.sht_quick_init | R.SHT_THETA_CONTIGUOUS, eps=0.0, nthreads=0)
    yield r
    r.close()


def test_highdeg_synthesis_against_long_double(plan):
    from oracle import sht_ld
    dev = torch.device("cuda:0")
    q = rand_spec(LMAX, LMAX, 1, 51, power=1.0)
    li, mi = lm_arrays(LMAX, LMAX, 1)
    rows = [0, 1, 2, 10, 600, 1200, 2400, 3071]
    phi_i = np.arange(0, NPHI, NPHI // 8)
    phi = 2 * np.pi * phi_i / NPHI
    for coeffs in (q, np.where(mi >= 2000, q, 0)):
        v = plan.synth(torch.from_numpy(coeffs).to(dev)).cpu().numpy()     # [nphi, nlat]
        vl = sht_ld.synth_points(coeffs, LMAX, plan.cos_theta[rows], phi).astype(float)
        err = np.abs(v[phi_i][:, rows].T - vl).max() / np.abs(v).max()
        assert err < 1e-11


def test_highdeg_against_reference(plan, ref):
    dev = torch.device("cuda:0")
    q = rand_spec(LMAX, LMAX, 1, 52, power=1.0)
    v = plan.synth(torch.from_numpy(q).to(dev)).cpu().numpy()
    vr = ref.synth(q)
    assert relerr(vr, v) < 1e-11
    qa = plan.analys(torch.from_numpy(vr).to(dev)).cpu().numpy()
    qr = ref.analys(vr)
    assert relerr(qr, qa) < 1e-11
    assert relerr(q, qa) < 1e-10


def test_highdeg_roundtrip_batch(plan):
    dev = torch.device("cuda:0")
    q = torch.from_numpy(rand_spec(LMAX, LMAX, 1, 53, power=1.0, nfields=2)).to(dev)
    back = plan.analys(plan.synth(q))
    assert float((back - q).abs().max() / q.abs().max()) < 1e-10
