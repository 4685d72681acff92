"""Seeded inputs shared by the tests, the golden-fixture generator and bench.py.

Spectral fields follow the input recipes of the benchmark configurations:
complex coefficients with N(0,1) real and imaginary parts scaled by
(l+1)^-p, imaginary part zero at m=0, optionally l=0 zeroed.  numpy's PCG64
generator makes them reproducible on any machine.
"""
import numpy as np


def lm_arrays(lmax, mmax, mres):
    li = np.concatenate([np.arange(im * mres, lmax + 1) for im in range(mmax + 1)])
    mi = np.concatenate([np.full(lmax + 1 - im * mres, im * mres) for im in range(mmax + 1)])
    return li, mi


def rand_spec(lmax, mmax, mres, seed, power=1.0, zero_l0=False, nfields=None, rng=None):
    """complex128 array [nfields, nlm] (or [nlm] if nfields is None)."""
    li, mi = lm_arrays(lmax, mmax, mres)
    rng = np.random.default_rng(seed) if rng is None else rng
    shape = (len(li),) if nfields is None else (nfields, len(li))
    q = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / (li + 1.0) ** power
    q = np.where(mi == 0, q.real + 0j, q)
    if zero_l0:
        q = np.where(li == 0, 0j, q)
    return np.ascontiguousarray(q)


def relerr(a, b):
    """max |a-b| / max |a| (normwise max relative error)."""
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.abs(a).max()
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))
