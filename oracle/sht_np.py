"""NumPy restatement of the SHTns 3.5.2 on-the-fly transform algorithm.

TEST INFRASTRUCTURE ONLY: the tests use it as the checker for the CUDA path
(next to the compiled reference library in oracle/_ref), __graft_entry__.smoke()
uses it at tiny size, and bench.py may time it as the CPU "port" baseline when
the reference library is absent.  The shtns_b200 product never imports it.

What it restates (reference file:line):
  * Gauss-Legendre nodes by Newton iteration on P_n, north pole first
    (sht_legendre.c:763-811), weights folded over the two hemispheres.
  * Associated Legendre recurrence with normalisation seeds (-1)^m*Y_00*
    sqrt(prod (2k+1)/(2k)) (sht_legendre.c:592-613) and coefficients
    a_l, b_l (sht_legendre.c:630-657), sin^m(theta) by binary powering with an
    extended exponent (sht_legendre.c:110-139) so that seeds below 1e-308 are
    carried instead of flushed to zero.
  * Synthesis v = sum_m (2-delta_m0) Re[F_m(theta) e^{i m phi}],
    F_m = sum_l Q_lm P_lm, with the equatorial symmetry P_lm(-x) =
    (-1)^(l+m) P_lm(x) folding north/south (kernel_SH_to_spat.gen.c:389-441).
  * Analysis by Gauss quadrature of the phi-Fourier coefficients
    (kernel_spat_to_SH.gen.c:485-598 with grid_weights in sht_init.c:560-649).
  * Vector transforms through two scalar transforms of V = sin(th) dS/dth +
    i m T and W = -sin(th) dT/dth + i m S divided by sin(th)
    (SH_vect_to_2scal, sht_private.h:534-584), and the inverse with the
    2cos+sin d/dth matrix and 1/(l(l+1)) (SH_2scal_to_vect,
    sht_private.h:296-337; matrices sht_func.c:400-447, sht_init.c:1378-1387).
  * Polar optimisation threshold: latitude rows where max_l |P_lm| < eps are
    treated as zero (PolarOptimize, sht_init.c:522-557).

Supported: Gauss grid, even nlat, orthonormal and 4pi normalisations with or
without Condon-Shortley phase and the real-norm option, mres >= 1, truncation
ltr <= lmax, theta- or phi-contiguous spatial layout.
"""
import numpy as np

# flag values from shtns.h:48-75
SHT_NO_CS_PHASE = 256 * 4
SHT_REAL_NORM = 256 * 8
SHT_THETA_CONTIGUOUS = 256
SHT_PHI_CONTIGUOUS = 256 * 2
SHT_SOUTH_POLE_FIRST = 256 * 32
sht_orthonormal, sht_fourpi, sht_schmidt = 0, 1, 2

_SCALE_BITS = 600          # extended exponent unit: values are y * 2^(600*e)


def gauss_nodes(n):
    """Gauss-Legendre nodes x (decreasing from +1) and weights, Newton on P_n
    from the asymptotic initial guess (sht_legendre.c:763-811), evaluated in
    extended precision (numpy longdouble) and rounded once."""
    LD = np.longdouble
    m = n // 2
    i = np.arange(m, dtype=LD)
    z = (LD(1) - LD(n - 1) / (LD(8) * n * n * n)) * np.cos(LD(np.pi) * (4 * i + 3) / LD(4 * n + 2))

    def legendre(z):
        p1 = z.copy()
        p2 = np.ones_like(z)
        for l in range(2, n + 1):
            p3 = p2
            p2 = p1
            p1 = ((2 * l - 1) * z * p2 - (l - 1) * p3) / l
        return p1, n * (p2 - z * p1)

    for _ in range(20):
        p1, pp = legendre(z)
        z1 = z
        z = z - p1 * (1 - z * z) / pp
        if np.all(np.abs(z - z1) <= (z1 + z) * LD(0.5) * LD(1e-19)):
            break
    p1, pp = legendre(z)
    s2 = (1 - z) * (1 + z)
    x = np.concatenate([z, -z[::-1]]).astype(np.float64)
    w = (2 * s2 / (pp * pp)).astype(np.float64)
    w = np.concatenate([w, w[::-1]])
    zr = z.astype(np.float64).astype(LD)                 # sin(theta) of the rounded node
    st = np.sqrt((1 - zr) * (1 + zr)).astype(np.float64)
    st = np.concatenate([st, st[::-1]])
    return x, st, w


class NpSHT:
    """Plan mirroring shtns_create(lmax, mmax, mres, norm) + shtns_set_grid on a
    Gauss grid.  Spectral arrays are complex128[..., nlm] in the LM order of
    shtns.h:104-106; spatial arrays are float64[..., nphi, nlat]
    (theta-contiguous) or [..., nlat, nphi] (phi-contiguous)."""

    def __init__(self, lmax, mmax=None, mres=1, norm=sht_orthonormal, nlat=None, nphi=None,
                 layout=SHT_THETA_CONTIGUOUS, eps=0.0):
        if mmax is None:
            mmax = lmax
        if mmax * mres > lmax:
            raise ValueError("mmax*mres > lmax")
        if nlat % 2:
            raise ValueError("odd nlat not supported by this restatement")
        if nlat <= lmax:
            raise ValueError("nlat must exceed lmax")
        if nphi <= 2 * mmax:
            raise ValueError("nphi must exceed 2*mmax")
        base = norm & 0xFF
        if base not in (sht_orthonormal, sht_fourpi):
            raise ValueError("restatement covers orthonormal and 4pi normalisations")
        self.lmax, self.mmax, self.mres = lmax, mmax, mres
        self.nlat, self.nphi = nlat, nphi
        self.norm = norm
        self.layout = layout
        self.cs = 0 if (norm & SHT_NO_CS_PHASE) else 1
        self.mpos_renorm = 0.5 if (norm & SHT_REAL_NORM) else 1.0
        self.base_norm = base
        x, st, w = gauss_nodes(nlat)
        if layout & SHT_SOUTH_POLE_FIRST:
            x = -x
        self.ct, self.st, self.wg = x, st, w
        self.nlat_2 = nlat // 2
        self.nlm = (mmax + 1) * (lmax + 1) - mres * mmax * (mmax + 1) // 2
        self.eps = eps
        self._seeds = self._seed_values()
        self._tm = self._polar_rows() if eps > 0 else np.zeros(mmax + 1, dtype=np.int64)

    # ---------------- indices and tables ----------------
    def idx(self, l, m):
        im = m // self.mres
        return (im * (2 * self.lmax + 2 - (im + 1) * self.mres)) // 2 + l

    def m_offset(self, im):
        return self.idx(im * self.mres, im * self.mres)

    def _seed_values(self):
        """Y_mm prefactors (sht_legendre.c:592-613), computed in long double."""
        if self.base_norm == sht_orthonormal:
            t1 = np.longdouble(0.25) / np.pi
        else:
            t1 = np.longdouble(1.0)
        seeds = np.zeros(self.mmax + 1)
        seeds[0] = float(np.sqrt(t1))
        t1 = t1 * np.longdouble(self.mpos_renorm)
        m = 0
        for im in range(1, self.mmax + 1):
            while m < im * self.mres:
                m += 1
                t1 *= (np.longdouble(m) + np.longdouble(0.5)) / np.longdouble(m)
            t2 = np.sqrt(t1)
            if (m & 1) and self.cs:
                t2 = -t2
            seeds[im] = float(t2)
        return seeds

    def _ab(self, m, lmax):
        """a_l, b_l for l = m..lmax (orthonormal / 4pi: sht_legendre.c:646-657)."""
        l = np.arange(m, lmax + 1, dtype=np.float64)
        a = np.zeros_like(l)
        b = np.zeros_like(l)
        if len(l) > 1:
            a[1] = np.sqrt(2.0 * m + 3.0)
        ll = l[2:]
        t1 = (ll + m) * (ll - m)
        a[2:] = np.sqrt((2 * ll + 1) * (2 * ll - 1) / t1)
        b[2:] = -np.sqrt((2 * ll + 1) * ((ll - 1 + m) * (ll - 1 - m)) / ((2 * ll - 3) * t1))
        return a, b

    def plm(self, im, lmax_p, x, st):
        """P_l^m(x) for l = m..lmax_p at the given nodes, shape [lmax_p-m+1, len(x)].
        Extended-exponent recurrence: values that never rise above 2^-600 return 0."""
        m = im * self.mres
        # sin^m by binary powering with exponent tracking (values y*2^(600 e))
        val = np.ones_like(x)
        ev = np.zeros(x.shape, dtype=np.int64)
        s2 = st.astype(np.float64).copy()
        es = np.zeros(x.shape, dtype=np.int64)
        n = m
        while n:
            if n & 1:
                val = val * s2
                ev = ev + es
                small = val < 2.0 ** -_SCALE_BITS
                val = np.where(small, np.ldexp(val, _SCALE_BITS), val)
                ev = ev - small
            n >>= 1
            if n:
                s2 = s2 * s2
                es = es + es
                small = s2 < 2.0 ** -_SCALE_BITS
                s2 = np.where(small, np.ldexp(s2, _SCALE_BITS), s2)
                es = es - small
        y0 = val * self._seeds[im]
        e = ev.copy()
        a, b = self._ab(m, lmax_p)
        nl = lmax_p - m + 1
        out = np.zeros((nl, len(x)))

        def emit(k, y):
            out[k] = np.where(e == 0, y, np.where(e < 0, np.ldexp(y, np.maximum(e, -4) * _SCALE_BITS), 0.0))

        emit(0, y0)
        if nl == 1:
            return out
        y1 = a[1] * x * y0
        emit(1, y1)
        for k in range(2, nl):
            y2 = a[k] * x * y1 + b[k] * y0
            y0, y1 = y1, y2
            big = (e < 0) & (np.abs(y1) > 1.0)
            if big.any():
                y0 = np.where(big, np.ldexp(y0, -_SCALE_BITS), y0)
                y1 = np.where(big, np.ldexp(y1, -_SCALE_BITS), y1)
                e = e + big
            emit(k, y1)
        return out

    def _polar_rows(self):
        """tm[im]: first north row where max_l |P_lm| >= eps (sht_init.c:522-557)."""
        tm = np.zeros(self.mmax + 1, dtype=np.int64)
        xs = np.abs(self.ct[: self.nlat_2])
        ss = self.st[: self.nlat_2]
        for im in range(1, self.mmax + 1):
            P = self.plm(im, self.lmax, np.abs(xs), ss)
            mx = np.abs(P).max(axis=0)
            ok = np.nonzero(mx >= self.eps)[0]
            tm[im] = ok[0] if len(ok) else self.nlat_2
        return tm

    # ---------------- layout helpers ----------------
    def _to_theta_phi(self, v):
        """spatial array -> [..., nlat, nphi]"""
        if self.layout & SHT_PHI_CONTIGUOUS:
            return v
        return np.swapaxes(v, -1, -2)

    def _from_theta_phi(self, g):
        if self.layout & SHT_PHI_CONTIGUOUS:
            return np.ascontiguousarray(g)
        return np.ascontiguousarray(np.swapaxes(g, -1, -2))

    def _north_P(self, im, lmax_p):
        n2 = self.nlat_2
        xs = np.abs(self.ct[:n2])   # |cos| of the north-hemisphere rows, decreasing
        P = self.plm(im, lmax_p, xs, self.st[:n2])
        P[:, : self._tm[im]] = 0.0
        return P

    def _row_order(self):
        """Map from stored rows to (north index, is_south): stored row t has
        |ct| at north index min(t, nlat-1-t)."""
        n2 = self.nlat_2
        t = np.arange(self.nlat)
        north = np.where(t < n2, t, self.nlat - 1 - t)
        south = t >= n2
        if self.layout & SHT_SOUTH_POLE_FIRST:
            south = ~south
        return north, south

    # ---------------- scalar-style Legendre stages ----------------
    def _legendre_synth(self, C, lmax_p, ltr, inv_sin):
        """C: dict im -> coefficients [..., lmax_p-m+1] (complex).  Returns the
        Fourier array [..., nlat, mmax_t+1] of F_m(theta)."""
        lead = next(iter(C.values())).shape[:-1]
        mmax_t = max(C.keys())
        F = np.zeros(lead + (self.nlat, mmax_t + 1), dtype=np.complex128)
        north, south = self._row_order()
        for im, c in C.items():
            m = im * self.mres
            P = self._north_P(im, lmax_p)              # [L, n2]
            L = c.shape[-1]
            P = P[:L]
            par = (np.arange(m, m + L) + m) % 2        # odd (l+m) changes sign in the south
            E = np.einsum("...l,lt->...t", c * (par == 0), P)
            O = np.einsum("...l,lt->...t", c * (par == 1), P)
            vals = np.where(south, E[..., north] - O[..., north], E[..., north] + O[..., north])
            if inv_sin:
                vals = vals / self.st[north]
            F[..., :, im] = vals
        return F

    def _fourier_to_spat(self, F):
        lead = F.shape[:-2]
        nc = self.nphi // 2 + 1
        G = np.zeros(lead + (self.nlat, nc), dtype=np.complex128)
        mm = min(F.shape[-1], nc)
        G[..., :mm] = F[..., :mm]
        g = np.fft.irfft(G, n=self.nphi, axis=-1) * self.nphi
        return self._from_theta_phi(g)

    def _spat_to_fourier(self, v, mmax_t):
        g = self._to_theta_phi(np.asarray(v, dtype=np.float64))
        G = np.fft.rfft(g, axis=-1) / self.nphi
        return G[..., : mmax_t + 1]

    def _quad_factor(self, m):
        """1/N_lm with N_lm = integral over x of P_lm^2 (orthonormal: 1/(2pi)
        times the real-norm factor for m>0; 4pi: 2 times that factor), times 2pi
        from the phi integral."""
        r = self.mpos_renorm if m > 0 else 1.0
        if self.base_norm == sht_orthonormal:
            return 2.0 * np.pi / r          # N_lm = r / (2 pi)
        return 0.5 / r                      # N_lm = 2 r

    def _legendre_analys(self, G, lmax_p, ltr, inv_sin):
        """G: [..., nlat, mmax_t+1] Fourier coefficients.  Returns dict im -> [..., L]."""
        north, south = self._row_order()
        n2 = self.nlat_2
        out = {}
        mmax_t = G.shape[-1] - 1
        for im in range(mmax_t + 1):
            m = im * self.mres
            if m > ltr:
                break
            P = self._north_P(im, lmax_p)               # [L, n2]
            w = self.wg[:n2].copy()
            g = G[..., im]
            if inv_sin:
                g = g / self.st
            # fold hemispheres: north row j pairs stored rows with north index j
            gn = np.zeros(g.shape[:-1] + (n2,), dtype=np.complex128)
            gs = np.zeros_like(gn)
            idx_n = np.nonzero(~south)[0]
            idx_s = np.nonzero(south)[0]
            gn[..., north[idx_n]] = g[..., idx_n]
            gs[..., north[idx_s]] = g[..., idx_s]
            ge = (gn + gs) * w
            go = (gn - gs) * w
            L = min(lmax_p, ltr if not inv_sin else ltr + 1) - m + 1
            par = (np.arange(m, m + L) + m) % 2
            qe = np.einsum("...t,lt->...l", ge, P[:L])
            qo = np.einsum("...t,lt->...l", go, P[:L])
            q = np.where(par == 0, qe, qo) * self._quad_factor(m)
            if m == 0:
                q = q.real.astype(np.complex128)
            out[im] = q
        return out

    # ---------------- public transforms ----------------
    def _mlim(self, ltr):
        return min(self.mmax, ltr // self.mres)

    def synth(self, q, ltr=None):
        """SH_to_spat / SH_to_spat_l (shtns.h:267,316)."""
        ltr = self.lmax if ltr is None else ltr
        q = np.asarray(q, dtype=np.complex128)
        C = {}
        for im in range(self._mlim(ltr) + 1):
            m = im * self.mres
            o = self.m_offset(im)
            c = q[..., o: o + (ltr - m + 1)].copy()
            if m == 0:
                c = c.real.astype(np.complex128)
            C[im] = c
        return self._fourier_to_spat(self._legendre_synth(C, self.lmax, ltr, False))

    def analys(self, v, ltr=None):
        """spat_to_SH / spat_to_SH_l (shtns.h:262,315)."""
        ltr = self.lmax if ltr is None else ltr
        v = np.asarray(v, dtype=np.float64)
        G = self._spat_to_fourier(v, self._mlim(ltr))
        Q = self._legendre_analys(G, self.lmax, ltr, False)
        out = np.zeros(v.shape[:-2] + (self.nlm,), dtype=np.complex128)
        for im, c in Q.items():
            o = self.m_offset(im)
            out[..., o: o + c.shape[-1]] = c
        return out

    def _alpha(self, m, lmax_p):
        """alpha_l = 1/a_l = sqrt((l^2-m^2)/((2l+1)(2l-1))) for l = m..lmax_p
        (cos(theta) coupling, sht_func.c:400-438); alpha_m = 0."""
        l = np.arange(m, lmax_p + 1, dtype=np.float64)
        al = np.zeros_like(l)
        k = l > m
        al[k] = np.sqrt((l[k] ** 2 - m * m) / ((2 * l[k] + 1) * (2 * l[k] - 1)))
        return al

    def sphtor_synth(self, s, t, ltr=None):
        """SHsphtor_to_spat (shtns.h:284): returns (Vt, Vp)."""
        ltr = self.lmax if ltr is None else ltr
        s = np.asarray(s, dtype=np.complex128)
        t = np.asarray(t, dtype=np.complex128)
        CV, CW = {}, {}
        for im in range(self._mlim(ltr) + 1):
            m = im * self.mres
            o = self.m_offset(im)
            L = ltr - m + 1
            S = np.zeros(s.shape[:-1] + (L + 3,), dtype=np.complex128)   # degrees m-1..ltr+2
            T = np.zeros_like(S)
            S[..., 1:L + 1] = s[..., o:o + L]
            T[..., 1:L + 1] = t[..., o:o + L]
            if m == 0:
                S = S.real.astype(np.complex128)
                T = T.real.astype(np.complex128)
            l = np.arange(m, ltr + 2, dtype=np.float64)          # output degrees m..ltr+1
            al = self._alpha(m, ltr + 2)                          # alpha_l for l = m..ltr+2
            # sin d/dth P_k = k alpha_{k+1} P_{k+1} - (k+1) alpha_k P_{k-1}
            # (stdt S)_l = (l-1) alpha_l S_{l-1} - (l+2) alpha_{l+1} S_{l+1}
            lo = (l - 1) * al[: L + 1]
            hi = -(l + 2) * al[1: L + 2]
            Sm1, Sp1 = S[..., 0:L + 1], S[..., 2:L + 3]
            Tm1, Tp1 = T[..., 0:L + 1], T[..., 2:L + 3]
            S0, T0 = S[..., 1:L + 2], T[..., 1:L + 2]
            CV[im] = lo * Sm1 + hi * Sp1 + 1j * m * T0
            CW[im] = -(lo * Tm1 + hi * Tp1) + 1j * m * S0
        Fv = self._legendre_synth(CV, self.lmax + 1, ltr, True)
        Fw = self._legendre_synth(CW, self.lmax + 1, ltr, True)
        return self._fourier_to_spat(Fv), self._fourier_to_spat(Fw)

    def sphtor_analys(self, vt, vp, ltr=None):
        """spat_to_SHsphtor (shtns.h:282): returns (Slm, Tlm)."""
        ltr = self.lmax if ltr is None else ltr
        mlim = self._mlim(ltr)
        Gv = self._spat_to_fourier(vt, mlim)
        Gw = self._spat_to_fourier(vp, mlim)
        A = self._legendre_analys(Gv, self.lmax + 1, ltr, True)    # degrees m..ltr+1
        B = self._legendre_analys(Gw, self.lmax + 1, ltr, True)
        lead = np.asarray(vt).shape[:-2]
        S = np.zeros(lead + (self.nlm,), dtype=np.complex128)
        T = np.zeros_like(S)
        for im in A:
            m = im * self.mres
            a, b = A[im], B[im]
            L = ltr - m + 1
            l = np.arange(m, ltr + 1, dtype=np.float64)
            al = self._alpha(m, ltr + 1)                           # l = m..ltr+1
            Am1 = np.concatenate([np.zeros(a.shape[:-1] + (1,)), a[..., :L - 1]], axis=-1)
            Bm1 = np.concatenate([np.zeros(b.shape[:-1] + (1,)), b[..., :L - 1]], axis=-1)
            Ap1, Bp1 = a[..., 1:L + 1], b[..., 1:L + 1]
            A0, B0 = a[..., :L], b[..., :L]
            c_lo = (l + 1) * al[:L]          # coefficient of X_{l-1}
            c_hi = l * al[1:L + 1]           # coefficient of X_{l+1}
            ll1 = l * (l + 1)
            inv = np.where(ll1 > 0, 1.0 / np.where(ll1 > 0, ll1, 1.0), 0.0)
            Sv = (c_hi * Ap1 - c_lo * Am1 - 1j * m * B0) * inv
            Tv = (-(c_hi * Bp1 - c_lo * Bm1) - 1j * m * A0) * inv
            o = self.m_offset(im)
            S[..., o:o + L] = Sv
            T[..., o:o + L] = Tv
            if m == 0:
                S[..., o:o + L] = Sv.real
                T[..., o:o + L] = Tv.real
        return S, T

    def qst_synth(self, q, s, t, ltr=None):
        """SHqst_to_spat (shtns.h:306)."""
        vr = self.synth(q, ltr)
        vt, vp = self.sphtor_synth(s, t, ltr)
        return vr, vt, vp

    def qst_analys(self, vr, vt, vp, ltr=None):
        """spat_to_SHqst (shtns.h:303)."""
        q = self.analys(vr, ltr)
        s, t = self.sphtor_analys(vt, vp, ltr)
        return q, s, t
