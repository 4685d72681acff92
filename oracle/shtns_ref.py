"""ctypes binding of the reference SHTns 3.5.2 CPU library built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY.  Used by the tests as the parity checker and by
bench.py's CPU-baseline leg and reference arm; the shtns_b200 product never
imports it.

The library is the reference's own C sources (sht_init.c, sht_kernels_[as].c,
sht_fly.c, sht_omp.c, sht_odd_nlat.c and the sed-generated SHT codelets)
compiled unchanged with OpenMP and Ishioka's recurrence, linked to the project's
FFTW-API shim.  Entry points bound here are the reference's public API
(shtns.h:149-324); argument meaning follows that header.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

# enum shtns_norm / shtns_type and layout flags (shtns.h:48-75)
sht_orthonormal, sht_fourpi, sht_schmidt = 0, 1, 2
SHT_NO_CS_PHASE = 256 * 4
SHT_REAL_NORM = 256 * 8
sht_gauss, sht_auto, sht_reg_fast, sht_reg_dct, sht_quick_init, sht_reg_poles, sht_gauss_fly = range(7)
SHT_NATIVE_LAYOUT = 0
SHT_THETA_CONTIGUOUS = 256
SHT_PHI_CONTIGUOUS = 256 * 2
SHT_SOUTH_POLE_FIRST = 256 * 32
SHT_SCALAR_ONLY = 256 * 16


class ShtnsInfo(C.Structure):
    """Public prefix of struct shtns_info (shtns.h:79-94)."""
    _fields_ = [
        ("nlm", C.c_uint),
        ("lmax", C.c_ushort),
        ("mmax", C.c_ushort),
        ("mres", C.c_ushort),
        ("nlat_2", C.c_ushort),
        ("nlat", C.c_uint),
        ("nphi", C.c_uint),
        ("nspat", C.c_uint),
        ("li", C.POINTER(C.c_ushort)),
        ("mi", C.POINTER(C.c_ushort)),
        ("ct", C.POINTER(C.c_double)),
        ("st", C.POINTER(C.c_double)),
        ("nlat_padded", C.c_uint),
        ("nlm_cplx", C.c_uint),
    ]


def _cpu_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = line.split()
                    return all(x in fl for x in ("avx512f", "avx512dq", "avx512bw", "avx512vl", "avx512cd"))
    except OSError:
        pass
    return False


_lib = None


def library_path():
    isa = "avx512" if _cpu_has_avx512() else "avx2"
    return os.path.join(REF_DIR, f"liboracle_shtns_{isa}.so")


def available():
    return os.path.exists(library_path())


def lib():
    """Load the reference library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise FileNotFoundError(f"reference oracle library missing: {path} (run make -C oracle)")
    L = C.CDLL(path)
    P = C.c_void_p
    cfg = C.POINTER(ShtnsInfo)
    dp = C.POINTER(C.c_double)
    L.shtns_create.restype = cfg
    L.shtns_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
    L.shtns_set_grid.restype = C.c_int
    L.shtns_set_grid.argtypes = [cfg, C.c_int, C.c_double, C.c_int, C.c_int]
    L.shtns_destroy.argtypes = [cfg]
    L.shtns_use_threads.restype = C.c_int
    L.shtns_use_threads.argtypes = [C.c_int]
    L.shtns_verbose.argtypes = [C.c_int]
    L.shtns_gauss_wts.restype = C.c_int
    L.shtns_gauss_wts.argtypes = [cfg, dp]
    L.nlm_calc.restype = C.c_long
    L.nlm_calc.argtypes = [C.c_long, C.c_long, C.c_long]
    L.SH_to_spat.argtypes = [cfg, P, P]
    L.spat_to_SH.argtypes = [cfg, P, P]
    L.SH_to_spat_l.argtypes = [cfg, P, P, C.c_int]
    L.spat_to_SH_l.argtypes = [cfg, P, P, C.c_int]
    L.SHsphtor_to_spat.argtypes = [cfg, P, P, P, P]
    L.spat_to_SHsphtor.argtypes = [cfg, P, P, P, P]
    L.SHsphtor_to_spat_l.argtypes = [cfg, P, P, P, P, C.c_int]
    L.spat_to_SHsphtor_l.argtypes = [cfg, P, P, P, P, C.c_int]
    L.SHqst_to_spat.argtypes = [cfg, P, P, P, P, P, P]
    L.spat_to_SHqst.argtypes = [cfg, P, P, P, P, P, P]
    L.SHqst_to_spat_l.argtypes = [cfg, P, P, P, P, P, P, C.c_int]
    L.spat_to_SHqst_l.argtypes = [cfg, P, P, P, P, P, P, C.c_int]
    L.SH_to_point.restype = C.c_double
    L.SH_to_point.argtypes = [cfg, P, C.c_double, C.c_double]
    L.legendre_sphPlm_array.restype = C.c_int
    L.legendre_sphPlm_array.argtypes = [cfg, C.c_int, C.c_int, C.c_double, dp]
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class RefSHT:
    """One reference plan: shtns_create + shtns_set_grid with theta-contiguous
    layout by default.  Arrays follow the reference layouts: spectral
    complex128[nlm] (LM index, shtns.h:104-106), spatial float64[nphi, nlat]
    for theta-contiguous data."""

    def __init__(self, lmax, mmax=None, mres=1, norm=sht_orthonormal, nlat=None, nphi=None,
                 flags=sht_gauss | SHT_THETA_CONTIGUOUS, eps=0.0, nthreads=1):
        L = lib()
        L.shtns_verbose(0)
        L.shtns_use_threads(int(nthreads))
        if mmax is None:
            mmax = lmax
        self.cfg = L.shtns_create(int(lmax), int(mmax), int(mres), int(norm))
        if not self.cfg:
            raise RuntimeError("shtns_create failed")
        self.nspat = L.shtns_set_grid(self.cfg, int(flags), float(eps), int(nlat), int(nphi))
        s = self.cfg.contents
        self.lmax, self.mmax, self.mres = s.lmax, s.mmax, s.mres
        self.nlm, self.nlat, self.nphi = s.nlm, s.nlat, s.nphi
        self.flags = flags
        self.ct = np.ctypeslib.as_array(s.ct, shape=(self.nlat,)).copy()
        self.st = np.ctypeslib.as_array(s.st, shape=(self.nlat,)).copy()
        self.li = np.ctypeslib.as_array(s.li, shape=(self.nlm,)).astype(np.int64)
        self.mi = np.ctypeslib.as_array(s.mi, shape=(self.nlm,)).astype(np.int64)
        self._L = L

    def spat_shape(self):
        if self.flags & SHT_PHI_CONTIGUOUS:
            return (self.nlat, self.nphi)
        return (self.nphi, self.nlat)

    def gauss_wts(self):
        w = np.zeros((self.nlat + 1) // 2)
        self._L.shtns_gauss_wts(self.cfg, w.ctypes.data_as(C.POINTER(C.c_double)))
        return w

    def idx(self, l, m):
        im = m // self.mres
        return (im * (2 * self.lmax + 2 - (im + 1) * self.mres)) // 2 + l

    def _spat(self):
        return np.zeros(self.spat_shape(), dtype=np.float64)

    def _spec(self):
        return np.zeros(self.nlm, dtype=np.complex128)

    def synth(self, q, ltr=None):
        q = np.ascontiguousarray(q, dtype=np.complex128)
        v = self._spat()
        if ltr is None:
            self._L.SH_to_spat(self.cfg, _p(q), _p(v))
        else:
            self._L.SH_to_spat_l(self.cfg, _p(q), _p(v), int(ltr))
        return v

    def analys(self, v, ltr=None):
        v = np.array(v, dtype=np.float64, order="C", copy=True)   # input may be overwritten
        q = self._spec()
        if ltr is None:
            self._L.spat_to_SH(self.cfg, _p(v), _p(q))
        else:
            self._L.spat_to_SH_l(self.cfg, _p(v), _p(q), int(ltr))
        return q

    def sphtor_synth(self, s, t, ltr=None):
        s = np.ascontiguousarray(s, dtype=np.complex128)
        t = np.ascontiguousarray(t, dtype=np.complex128)
        vt, vp = self._spat(), self._spat()
        if ltr is None:
            self._L.SHsphtor_to_spat(self.cfg, _p(s), _p(t), _p(vt), _p(vp))
        else:
            self._L.SHsphtor_to_spat_l(self.cfg, _p(s), _p(t), _p(vt), _p(vp), int(ltr))
        return vt, vp

    def sphtor_analys(self, vt, vp, ltr=None):
        vt = np.array(vt, dtype=np.float64, order="C", copy=True)
        vp = np.array(vp, dtype=np.float64, order="C", copy=True)
        s, t = self._spec(), self._spec()
        if ltr is None:
            self._L.spat_to_SHsphtor(self.cfg, _p(vt), _p(vp), _p(s), _p(t))
        else:
            self._L.spat_to_SHsphtor_l(self.cfg, _p(vt), _p(vp), _p(s), _p(t), int(ltr))
        return s, t

    def qst_synth(self, q, s, t, ltr=None):
        q, s, t = (np.ascontiguousarray(a, dtype=np.complex128) for a in (q, s, t))
        vr, vt, vp = self._spat(), self._spat(), self._spat()
        if ltr is None:
            self._L.SHqst_to_spat(self.cfg, _p(q), _p(s), _p(t), _p(vr), _p(vt), _p(vp))
        else:
            self._L.SHqst_to_spat_l(self.cfg, _p(q), _p(s), _p(t), _p(vr), _p(vt), _p(vp), int(ltr))
        return vr, vt, vp

    def qst_analys(self, vr, vt, vp, ltr=None):
        vr, vt, vp = (np.array(a, dtype=np.float64, order="C", copy=True) for a in (vr, vt, vp))
        q, s, t = self._spec(), self._spec(), self._spec()
        if ltr is None:
            self._L.spat_to_SHqst(self.cfg, _p(vr), _p(vt), _p(vp), _p(q), _p(s), _p(t))
        else:
            self._L.spat_to_SHqst_l(self.cfg, _p(vr), _p(vt), _p(vp), _p(q), _p(s), _p(t), int(ltr))
        return q, s, t

    def point(self, q, cost, phi):
        q = np.ascontiguousarray(q, dtype=np.complex128)
        return self._L.SH_to_point(self.cfg, _p(q), float(cost), float(phi))

    def plm_array(self, m, x, lmax=None):
        """legendre_sphPlm_array (shtns.h:215): P_l^m(x) for l=m..lmax."""
        if lmax is None:
            lmax = self.lmax
        y = np.zeros(lmax - m + 1)
        self._L.legendre_sphPlm_array(self.cfg, int(lmax), int(m // self.mres), float(x),
                                      y.ctypes.data_as(C.POINTER(C.c_double)))
        return y

    def close(self):
        if self.cfg:
            self._L.shtns_destroy(self.cfg)
            self.cfg = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
