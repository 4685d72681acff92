"""Long-double evaluation of scalar synthesis at selected latitudes (test
infrastructure: an accuracy reference for high degrees, not a product path).

For a few latitude nodes x = cos(theta) (given as doubles: the same inputs
the transforms see) and longitudes phi, evaluates

    v(theta, phi) = sum_m sum_{l>=m} Q_lm P_lm(x) e^{i m phi}   (real part, m>0 doubled)

with orthonormal, Condon-Shortley-phased P_lm computed by the classical
three-term recurrence in l (sht_legendre.c:592-657: seeds
Y_mm = (-1)^m sqrt((2m+1)!!/((2m)!! 4 pi)) sin^m theta, a_l, b_l of the
orthonormal recurrence), vectorised over m, in numpy longdouble (64-bit
mantissa on x86, exponent range to 1e-4951, so no scaling is needed up to
degree 4095 except at the few rows closest to the poles, whose values
underflow to exact zeros far below any significant term).

Rounding of this evaluation is ~1e-16 relative, four orders below the errors
it is used to measure.
"""
import numpy as np

LD = np.longdouble


def _seeds(mmax):
    """(-1)^m sqrt((2m+1)!!/((2m)!! 4pi)) for m = 0..mmax in long double."""
    t = LD(0.25) / LD(np.pi)
    out = np.empty(mmax + 1, dtype=LD)
    out[0] = np.sqrt(t)
    for m in range(1, mmax + 1):
        t *= (LD(m) + LD(0.5)) / LD(m)
        out[m] = np.sqrt(t) * (-1 if m & 1 else 1)
    return out


def legendre_sums(q, lmax, x, st=None):
    """G[m] = sum_l Q_lm P_lm(x) for m = 0..lmax at one node x (mmax = lmax,
    mres = 1, SHTns l-within-m coefficient order).  Returns complex long double.
    sin(theta) is sqrt(1 - x^2) of the given x unless st is given."""
    xl = LD(x)
    st = np.sqrt((LD(1) - xl) * (LD(1) + xl)) if st is None else LD(st)
    m = np.arange(lmax + 1)
    ml = m.astype(LD)
    off = (m * (2 * lmax + 3 - m)) // 2 - m            # index of (l, m) = off[m] + l
    qr = np.asarray(q.real, dtype=LD)
    qi = np.asarray(q.imag, dtype=LD)
    # P_mm = seed * sin^m (pow in long double; may underflow to 0 near the poles)
    p0 = _seeds(lmax) * st ** ml
    gr = p0 * qr[off + m]
    gi = p0 * qi[off + m]
    # P_{m+1,m} = sqrt(2m+3) x P_mm
    sel = m + 1 <= lmax
    p1 = np.zeros_like(p0)
    p1[sel] = np.sqrt(LD(2) * ml[sel] + LD(3)) * xl * p0[sel]
    gr[sel] += p1[sel] * qr[off[sel] + m[sel] + 1]
    gi[sel] += p1[sel] * qi[off[sel] + m[sel] + 1]
    pm2, pm1 = p0, p1
    for j in range(2, lmax + 1):
        n = lmax + 1 - j                                # orders with m + j <= lmax
        mm = ml[:n]
        l = mm + LD(j)
        t1 = (l + mm) * (l - mm)
        a = np.sqrt((LD(2) * l + 1) * (LD(2) * l - 1) / t1)
        b = -np.sqrt((LD(2) * l + 1) * ((l - 1 + mm) * (l - 1 - mm)) / ((LD(2) * l - 3) * t1))
        p = a * xl * pm1[:n] + b * pm2[:n]
        idx = off[:n] + m[:n] + j
        gr[:n] += p * qr[idx]
        gi[:n] += p * qi[idx]
        pm2, pm1 = pm1[:n], p
    return gr + 1j * gi


def synth_points(q, lmax, x, phi, st=None):
    """v at the nodes x (sequence of doubles) and longitudes phi (array):
    returns long double array [len(x), len(phi)].  st: optional sin(theta)
    of each node (default sqrt(1 - x^2))."""
    phi = np.asarray(phi, dtype=LD)
    m = np.arange(lmax + 1, dtype=LD)
    ang = np.outer(phi, m)
    c, s = np.cos(ang), np.sin(ang)
    out = np.empty((len(x), len(phi)), dtype=LD)
    for i, xv in enumerate(x):
        g = legendre_sums(q, lmax, xv, None if st is None else st[i])
        gr, gi = g.real.astype(LD), g.imag.astype(LD)
        fac = np.full(lmax + 1, LD(2))
        fac[0] = LD(1)
        out[i] = (c * (fac * gr)).sum(axis=1) - (s * (fac * gi)).sum(axis=1)
    return out
