"""CPU check of the index mapping of the FFT analysis's last pass
(sht_fft.cu, last_pass_pairs): with nphi = N = 3 P, the radix-3 butterfly b
(b < P) produces z_{b + q P}, q = 0, 1, 2.  A thread that runs butterflies b
and P - b holds both members of (z_k, z_{N-k}) for k = b, P - b, P + b
(b = 0: k = 0, P; b = P/2: k = P/2).  Over b = 0 .. P/2 every k < N/2 is
handed over exactly once, with its partner; the Fourier rows then follow as
F_k = (z_k + conj z_{N-k}) / (2N) for the first latitude of the pair and
(z_k - conj z_{N-k}) / (2iN) for the second, as np.fft gives them."""
import numpy as np
import pytest


def pairs(N):
    P = N // 3
    H = P // 2
    out = []
    for b in range(H + 1):
        u = [b + q * P for q in range(3)]                 # outputs of butterfly b
        if b == 0:
            out += [(0, u[0], u[0]), (P, u[1], u[2])]
        elif b == H:
            out += [(H, u[0], u[2])]
        else:
            v = [P - b + q * P for q in range(3)]         # outputs of butterfly P - b
            out += [(b, u[0], v[2]), (P - b, v[0], u[2]), (P + b, u[1], v[1])]
    return out


@pytest.mark.parametrize("N", [192, 384, 768, 1536, 3072, 6144, 12288])
def test_pairs_cover_every_order_once_with_its_partner(N):
    pr = pairs(N)
    ks = sorted(k for k, _, _ in pr)
    assert ks == list(range(N // 2))
    for k, i, j in pr:
        assert i == k and j == (N - k) % N


@pytest.mark.parametrize("N", [192, 1536])
def test_fourier_rows_from_pairs_match_numpy(N):
    rng = np.random.default_rng(N)
    va, vb = rng.standard_normal(N), rng.standard_normal(N)    # two latitudes
    # the kernel's analysis DFT has sign -1: z_k = sum_j (va + i vb)_j e^{-2 pi i jk/N}
    z = np.fft.fft(va + 1j * vb)
    fa, fb = np.fft.fft(va) / N, np.fft.fft(vb) / N
    for k, i, j in pairs(N):
        zk, wk = z[i], z[j]
        a = 0.5 / N * complex(zk.real + wk.real, zk.imag - wk.imag)
        b = 0.5 / N * complex(zk.imag + wk.imag, -(zk.real - wk.real))
        assert abs(a - fa[k]) < 1e-12 and abs(b - fb[k]) < 1e-12
