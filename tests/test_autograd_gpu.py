"""Differentiable transforms (torch.autograd) with hand-written adjoint kernels.

Configuration: lmax=255, Gauss 384 x 768, batch 128, FP64 and FP32.  Loss
L = sum_grid w_j (u^2 - u0^2)^2 with u = synth(q), w_j the Gauss weight of
the latitude, u0 a seeded target field.  Checks:
  * adjointness: <g, S q> = <S^T g, q> and <h, A v> = <A^T h, v> (real inner
    products, complex numbers as pairs of reals) to rounding;
  * the autograd gradient equals the gradient built from the reference's own
    analysis / synthesis (S^T g = (2 - delta_m0) nphi / (2 pi) A(g / w_theta),
    A^T h = 2 pi w_theta / nphi S(h with m>0 halved)) to 1e-10 relative;
  * central finite differences (h = 1e-6, FP64) along random directions;
  * FP32 gradients agree with FP64 ones to FP32 accuracy.
"""
import numpy as np
import pytest

from tests.common import rand_spec, relerr, lm_arrays

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

LMAX, NLAT, NPHI, NB = 255, 384, 768, 128


@pytest.fixture(scope="module")
def plan():
    import shtns_b200
    sh = shtns_b200.sht(LMAX)
    sh.set_grid(NLAT, NPHI, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=0.0)
    return sh


def _rdot(a, b):
    """real inner product of two tensors (complex as pairs of reals)"""
    if a.is_complex():
        return float((a.real * b.real + a.imag * b.imag).sum())
    return float((a * b).sum())


def _weights(sh, dev, dtype=torch.float64):
    w = np.concatenate([sh.gauss_wts(), sh.gauss_wts()[::-1]])      # per latitude, north first
    return torch.from_numpy(w).to(dev, dtype)                       # broadcast over phi (theta last)


def test_adjoint_dot_products(plan):
    from shtns_b200 import autograd as ad
    dev = torch.device("cuda:0")
    q = torch.from_numpy(rand_spec(LMAX, LMAX, 1, 1, nfields=4)).to(dev)
    g = torch.randn((4,) + plan.spat_shape, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(2))
    # synthesis
    qq = q.clone().requires_grad_(True)
    v = ad.synth(plan, qq)
    (v * g).sum().backward()
    lhs, rhs = _rdot(g, v.detach()), _rdot(qq.grad, q)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0) * 1e2
    # analysis
    h = torch.from_numpy(rand_spec(LMAX, LMAX, 1, 3, nfields=4)).to(dev)
    vv = g.clone().requires_grad_(True)
    Q = ad.analys(plan, vv)
    (h.real * Q.real + h.imag * Q.imag).sum().backward()
    lhs, rhs = _rdot(h, Q.detach()), _rdot(vv.grad, g)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0) * 1e2


def _loss(u, u0, w):
    return (w * (u * u - u0 * u0) ** 2).sum()


def test_cfg4_gradient_against_reference_transforms(plan):
    from oracle import shtns_ref as R
    if not R.available():
        pytest.skip("reference library not built")
    from shtns_b200 import autograd as ad
    dev = torch.device("cuda:0")
    qn = rand_spec(LMAX, LMAX, 1, 10, nfields=NB)
    q = torch.from_numpy(qn).to(dev).requires_grad_(True)
    u0 = ad.synth(plan, torch.from_numpy(rand_spec(LMAX, LMAX, 1, 11, nfields=NB)).to(dev)).detach()
    w = _weights(plan, dev)
    u = ad.synth(plan, q)
    L = _loss(u, u0, w)
    L.backward()
    # gradient built from the reference's own transforms
    ref = R.RefSHT(LMAX, LMAX, 1, R.sht_orthonormal, NLAT, NPHI, flags=R.sht_quick_init | R.SHT_THETA_CONTIGUOUS, eps=0.0, nthreads=16)
    un, u0n, wn = u.detach().cpu().numpy(), u0.cpu().numpy(), w.cpu().numpy()
    dLdu = 4.0 * wn * (un * un - u0n * u0n) * un                    # [NB, nphi, nlat]
    li, mi = lm_arrays(LMAX, LMAX, 1)
    fac = np.where(mi == 0, 1.0, 2.0) * NPHI / (2 * np.pi)
    gref = np.stack([fac * ref.analys(dLdu[f] / wn) for f in range(NB)])
    gref[:, mi == 0] = gref[:, mi == 0].real
    assert relerr(gref, q.grad.cpu().numpy()) < 1e-10
    ref.close()


def test_analysis_adjoint_against_reference_transforms(plan):
    from oracle import shtns_ref as R
    if not R.available():
        pytest.skip("reference library not built")
    from shtns_b200 import autograd as ad
    dev = torch.device("cuda:0")
    nf = 8
    v = ad.synth(plan, torch.from_numpy(rand_spec(LMAX, LMAX, 1, 20, nfields=nf)).to(dev)).detach().requires_grad_(True)
    hn = rand_spec(LMAX, LMAX, 1, 21, nfields=nf)
    h = torch.from_numpy(hn).to(dev)
    Q = ad.analys(plan, v)
    (h.real * Q.real + h.imag * Q.imag).sum().backward()
    ref = R.RefSHT(LMAX, LMAX, 1, R.sht_orthonormal, NLAT, NPHI, flags=R.sht_quick_init | R.SHT_THETA_CONTIGUOUS, eps=0.0, nthreads=16)
    li, mi = lm_arrays(LMAX, LMAX, 1)
    wrow = np.concatenate([plan.gauss_wts(), plan.gauss_wts()[::-1]])
    hh = np.where(mi == 0, hn.real + 0j, hn / 2)
    gref = np.stack([2 * np.pi * wrow / NPHI * ref.synth(hh[f]) for f in range(nf)])
    assert relerr(gref, v.grad.cpu().numpy()) < 1e-10
    ref.close()


def test_cfg4_gradient_finite_differences(plan):
    from shtns_b200 import autograd as ad
    dev = torch.device("cuda:0")
    q = torch.from_numpy(rand_spec(LMAX, LMAX, 1, 30, nfields=NB)).to(dev).requires_grad_(True)
    u0 = ad.synth(plan, torch.from_numpy(rand_spec(LMAX, LMAX, 1, 31, nfields=NB)).to(dev)).detach()
    w = _weights(plan, dev)
    L = _loss(ad.synth(plan, q), u0, w)
    L.backward()
    gen = torch.Generator(dev).manual_seed(5)
    h = 1e-6
    for _ in range(3):
        d = torch.randn(q.shape, dtype=torch.complex128, device=dev, generator=gen)
        d[:, : LMAX + 1] = d[:, : LMAX + 1].real + 0j                # m=0 coefficients are real
        d = d / torch.sqrt((d.real ** 2 + d.imag ** 2).sum())
        with torch.no_grad():
            lp = _loss(ad.synth(plan, q + h * d), u0, w)
            lm = _loss(ad.synth(plan, q - h * d), u0, w)
        fd = float((lp - lm) / (2 * h))
        an = _rdot(q.grad, d)
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-9 * float(L.detach())


def test_fp32_gradients_match_fp64(plan):
    from shtns_b200 import autograd as ad
    dev = torch.device("cuda:0")
    qn = rand_spec(LMAX, LMAX, 1, 40, nfields=NB)
    u0 = ad.synth(plan, torch.from_numpy(rand_spec(LMAX, LMAX, 1, 41, nfields=NB)).to(dev)).detach()
    grads = {}
    for dt, ct in ((torch.float64, torch.complex128), (torch.float32, torch.complex64)):
        q = torch.from_numpy(qn).to(dev, ct).requires_grad_(True)
        u = ad.synth(plan, q)
        assert u.dtype == dt
        L = _loss(u, u0.to(dt), _weights(plan, dev, dt))
        L.backward()
        grads[dt] = q.grad.to(torch.complex128).cpu().numpy()
    assert relerr(grads[torch.float64], grads[torch.float32]) < 1e-4
