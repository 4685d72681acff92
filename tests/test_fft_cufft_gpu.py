"""The library's own phi-FFT kernels (sht_fft.cu) against cuFFT.

The Fourier side of the transform holds, for each grid row theta and order
m <= mmax, F_m(theta) = (1/nphi) sum_j v(theta, phi_j) exp(-2 pi i m j / nphi)
(analysis), and the synthesis is v(theta, phi_j) = sum_m (2 - delta_m0)
Re[F_m(theta) exp(2 pi i m j / nphi)].  cuFFT computes the same with the
reference's packing (sht_gpu.cu:186-190): latitude pairs (2p, 2p+1) as the
real and imaginary parts of one complex sequence, a Z2Z transform of length
nphi over the nlat/2 pairs, and the two real spectra separated afterwards.

Both directions are compared through the order-split stage entry points
shtns_b200_fourier_analys / shtns_b200_fourier_synth (the FFT stage alone),
at nphi = 192, 1536, 3072 (every grid row) and 12288 (a block of 64 rows),
on theta-contiguous grids; bar 1e-13 normwise."""
import ctypes as C

import numpy as np
import pytest
import torch

from tests.common import relerr

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _plan(nphi):
    import shtns_b200
    lmax = nphi // 3 - 1
    sh = shtns_b200.sht(lmax)
    sh.set_grid(nphi // 2, nphi, flags=shtns_b200.sht_quick_init | shtns_b200.SHT_THETA_CONTIGUOUS, polar_opt=0.0)
    return sh


def _cufft_pairs(v, direction):
    """v: [nphi][nrows] float64 (theta-contiguous).  Forward: X[k][p], the Z2Z
    transform (sign -1) of the latitude-pair sequences, through the reference's
    cuFFT plan.  Inverse: the same with sign +1."""
    from tests import cufft
    nphi, nrows = v.shape
    z = v.contiguous().view(torch.complex128).clone()          # [nphi][nrows/2]
    plan = cufft.PairPlan(nphi, nrows, torch.cuda.current_stream().cuda_stream)
    plan.exec(z.data_ptr(), z.data_ptr(), direction)
    torch.cuda.synchronize()
    plan.destroy()
    return z


@pytest.mark.parametrize("nphi,nrows", [(192, 0), (1536, 0), (3072, 0), (12288, 64)])
def test_fourier_analysis_matches_cufft(nphi, nrows):
    from shtns_b200 import capi
    lib = capi.load()
    sh = _plan(nphi)
    nrows = nrows or sh.nlat
    mmax = sh.mmax
    dev = torch.device("cuda:0")
    g = torch.Generator(device="cpu").manual_seed(nphi)
    v = torch.randn((nphi, nrows), dtype=torch.float64, generator=g).to(dev)
    F = torch.zeros((mmax + 1, nrows), dtype=torch.complex128, device=dev)
    lib.shtns_set_batch(sh._cfg, 1, sh.nlm, sh.nspat)
    lib.cushtns_set_streams(sh._cfg, C.c_void_p(torch.cuda.current_stream().cuda_stream), None)
    lib.shtns_b200_status()
    lib.shtns_b200_fourier_analys(sh._cfg, 0, C.c_void_p(v.data_ptr()), None, None, C.c_void_p(F.data_ptr()),
                                  nrows, sh.lmax)
    torch.cuda.synchronize()
    assert lib.shtns_b200_status() == 0, lib.shtns_b200_last_error().decode()
    X = _cufft_pairs(v, -1)                                     # [nphi][nrows/2]
    k = torch.arange(mmax + 1, device=dev)
    Xk, Xn = X[k], X[(-k) % nphi].conj()
    want = torch.empty((mmax + 1, nrows), dtype=torch.complex128, device=dev)
    want[:, 0::2] = (Xk + Xn) / (2 * nphi)
    want[:, 1::2] = (Xk - Xn) / (2j * nphi)
    assert relerr(want.cpu().numpy(), F.cpu().numpy()) < TOL
    # and the plain real DFT of each row (torch.fft, also cuFFT)
    R = torch.fft.rfft(v, dim=0)[: mmax + 1] / nphi
    assert relerr(R.cpu().numpy(), F.cpu().numpy()) < TOL


@pytest.mark.parametrize("nphi,nrows", [(192, 0), (1536, 0), (3072, 0), (12288, 64)])
def test_fourier_synthesis_matches_cufft(nphi, nrows):
    from shtns_b200 import capi
    lib = capi.load()
    sh = _plan(nphi)
    nrows = nrows or sh.nlat
    mmax = sh.mmax
    dev = torch.device("cuda:0")
    g = torch.Generator(device="cpu").manual_seed(nphi + 1)
    F = torch.randn((mmax + 1, nrows), dtype=torch.complex128, generator=g)
    F[0] = F[0].real.to(torch.complex128)                      # m = 0 rows are real
    F = F.to(dev)
    v = torch.full((nphi, nrows), float("nan"), dtype=torch.float64, device=dev)
    lib.shtns_set_batch(sh._cfg, 1, sh.nlm, sh.nspat)
    lib.cushtns_set_streams(sh._cfg, C.c_void_p(torch.cuda.current_stream().cuda_stream), None)
    lib.shtns_b200_status()
    lib.shtns_b200_fourier_synth(sh._cfg, 0, C.c_void_p(F.data_ptr()), C.c_void_p(v.data_ptr()), None, None,
                                 nrows, sh.lmax)
    torch.cuda.synchronize()
    assert lib.shtns_b200_status() == 0, lib.shtns_b200_last_error().decode()
    # pair spectra Z_k = A_k + i B_k, Z_{N-k} = conj(A_k) + i conj(B_k), then the inverse Z2Z through cuFFT
    Z = torch.zeros((nphi, nrows // 2), dtype=torch.complex128, device=dev)
    A, B = F[:, 0::2], F[:, 1::2]
    Z[: mmax + 1] = A + 1j * B
    k = torch.arange(1, mmax + 1, device=dev)
    Z[nphi - k] = A[1:].conj() + 1j * B[1:].conj()
    z = _cufft_pairs(torch.view_as_real(Z).reshape(nphi, nrows), +1)
    want = torch.view_as_real(z).reshape(nphi, nrows)
    got = v.cpu().numpy()
    assert np.isfinite(got).all()
    assert relerr(want.cpu().numpy(), got) < TOL
