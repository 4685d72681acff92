"""Python surface of shtns_b200, mirroring the reference's `shtns.sht` class
(shtns_numpy.i:150-460): same constructor, set_grid, idx, spec_array,
spat_array, synth and analys semantics.

Arrays may be NumPy arrays (transformed through the host-pointer C API with
copies to and from the GPU) or torch CUDA tensors (transformed in place on the
device through the cu_* C API, on torch's current stream).  Leading dimensions
are batch dimensions: a spectral array of shape (..., nlm) or a spatial array
of shape (..., *spat_shape) transforms every field in one call.
"""
import ctypes as C

import numpy as np

from . import capi
from .capi import (sht_orthonormal, sht_fourpi, sht_schmidt, SHT_NO_CS_PHASE, SHT_REAL_NORM,  # noqa: F401
                   sht_gauss, sht_auto, sht_quick_init, sht_gauss_fly, sht_reg_fast, sht_reg_dct, sht_reg_poles,
                   SHT_NATIVE_LAYOUT, SHT_THETA_CONTIGUOUS, SHT_PHI_CONTIGUOUS, SHT_SOUTH_POLE_FIRST,
                   SHT_SCALAR_ONLY, SHT_LOAD_SAVE_CFG, SHT_ALLOW_GPU, SHT_ALLOW_PADDING, SHTError)

try:
    import torch
except ImportError:  # torch is optional for the NumPy path
    torch = None


def _is_torch(x):
    return torch is not None and isinstance(x, torch.Tensor)


class sht:
    """Spherical harmonic transform plan on the GPU.

    sht(lmax, mmax=-1, mres=1, norm=sht_orthonormal, nthreads=0) as in the
    reference (shtns_numpy.i:173-190); nthreads is accepted and ignored."""

    def __init__(self, lmax, mmax=-1, mres=1, norm=sht_orthonormal, nthreads=0):
        self._lib = capi.load()
        if lmax < 2:
            raise ValueError("lmax < 2 not allowed")
        if mres <= 0:
            raise ValueError("mres <= 0 invalid")
        if mmax < 0:
            mmax = lmax // mres
        if mmax * mres > lmax:
            raise ValueError("lmax < mmax*mres invalid")
        self._cfg = self._lib.shtns_create(int(lmax), int(mmax), int(mres), int(norm))
        if not self._cfg:
            raise SHTError(self._lib.shtns_b200_last_error().decode())
        s = self._cfg.contents
        self.lmax, self.mmax, self.mres, self.nlm = s.lmax, s.mmax, s.mres, s.nlm
        self.norm = norm
        self.nlat = 0
        self.nphi = 0
        self.l = np.zeros(self.nlm, dtype=np.int32)
        self.m = np.zeros(self.nlm, dtype=np.int32)
        for mm in range(0, self.mmax * self.mres + 1, self.mres):
            for ll in range(mm, self.lmax + 1):
                ii = self.idx(ll, mm)
                self.l[ii] = ll
                self.m[ii] = mm
        self.l.flags.writeable = False
        self.m.flags.writeable = False

    # ---------------- set-up ----------------
    def set_grid(self, nlat=0, nphi=0, flags=sht_quick_init, polar_opt=1.0e-10, nl_order=1):
        """Gauss grid set-up (shtns_numpy.i:204-222): default layout is
        phi-contiguous unless SHT_THETA_CONTIGUOUS is given."""
        if nlat != 0 and nlat <= self.lmax:
            raise ValueError("nlat <= lmax")
        if nphi != 0 and nphi <= self.mmax * 2:
            raise ValueError("nphi <= 2*mmax")
        if not (flags & SHT_THETA_CONTIGUOUS):
            flags |= SHT_PHI_CONTIGUOUS
        grd = flags & 255
        if grd in (sht_auto, sht_gauss_fly, sht_gauss):
            grd = sht_quick_init
        flags = (flags & ~255) | grd
        nl = C.c_int(int(nlat))
        np_ = C.c_int(int(nphi))
        r = self._lib.shtns_set_grid_auto(self._cfg, int(flags), float(polar_opt), int(nl_order),
                                          C.byref(nl), C.byref(np_))
        if r < 0:
            raise SHTError(self._lib.shtns_b200_last_error().decode())
        s = self._cfg.contents
        self.nlat, self.nphi, self.nspat = s.nlat, s.nphi, s.nspat
        self.flags = flags
        self.layout = flags & ~255
        self.cos_theta = np.ctypeslib.as_array(s.ct, shape=(self.nlat,)).copy()
        self.cos_theta.flags.writeable = False
        if self.layout & SHT_PHI_CONTIGUOUS:
            self.spat_shape = (self.nlat, self.nphi)
        else:
            self.spat_shape = (self.nphi, self.nlat)
        return self.nlat, self.nphi

    def robert_form(self, v=1):
        self._lib.shtns_robert_form(self._cfg, int(v))

    def print_info(self):
        self._lib.shtns_print_cfg(self._cfg)

    def sh00_1(self):
        return self._lib.sh00_1(self._cfg)

    def sh10_ct(self):
        return self._lib.sh10_ct(self._cfg)

    def sh11_st(self):
        return self._lib.sh11_st(self._cfg)

    def shlm_e1(self, l, m):
        return self._lib.shlm_e1(self._cfg, int(l), int(m))

    def gauss_wts(self):
        w = np.zeros(self.nlat // 2)
        n = self._lib.shtns_gauss_wts(self._cfg, w.ctypes.data_as(C.c_void_p))
        return w[:n]

    def idx(self, l, m):
        if l > self.lmax:
            raise ValueError("l invalid")
        if m > l or m > self.mmax * self.mres or m % self.mres != 0:
            raise ValueError("m invalid")
        im = m // self.mres
        return (im * (2 * self.lmax + 2 - (im + 1) * self.mres)) // 2 + l

    def spec_array(self, im=-1):
        if im < 0:
            return np.zeros(self.nlm, dtype=complex)
        return np.zeros(self.lmax + 1 - im * self.mres, dtype=complex)

    def spat_array(self):
        if self.nlat == 0:
            raise RuntimeError("Grid not set. Call .set_grid() method.")
        return np.zeros(self.spat_shape)

    def clone(self, stream=0):
        """cushtns_clone: a plan sharing this plan's tables, for another stream."""
        c = object.__new__(sht)
        c.__dict__.update(self.__dict__)
        c._cfg = self._lib.cushtns_clone(self._cfg, C.c_void_p(stream), None)
        if not c._cfg:
            raise SHTError(self._lib.shtns_b200_last_error().decode())
        c._clone_of = self
        return c

    def set_split(self, nslices, form=0):
        """Split-precision Legendre stages with `nslices` (3 to 7) 8-bit digits
        per operand; 0 restores the FP64 contraction.  form 0 (default): a
        precomputed table of the Legendre values as INT8 digits, contracted on
        the INT8 tensor cores with exact INT32 accumulation, for synthesis and
        analysis (the table, about nslices bytes per latitude, order and
        degree pair, is built on first use); form 1: synthesis only, slices
        regenerated on the fly and contracted on the FP16 tensor cores
        (analysis in FP64)."""
        if form not in (0, 1):
            raise ValueError("form must be 0 or 1")
        if self._lib.shtns_b200_set_option(self._cfg, 4, int(nslices)) != 0:
            raise ValueError("nslices must be 0 or 3..7")
        self._lib.shtns_b200_set_option(self._cfg, 8, int(form))

    def kernel_errors(self):
        """1 if a bounded wait inside a split-precision kernel gave up (the
        result of that call is not valid), else 0; clears the flag."""
        return self._lib.shtns_b200_kernel_errors(self._cfg)

    def device_bytes(self):
        return self._lib.shtns_b200_device_bytes(self._cfg)

    def __del__(self):
        try:
            if getattr(self, "_cfg", None):
                self._lib.shtns_destroy(self._cfg)
                self._cfg = None
        except Exception:
            pass

    # ---------------- helpers ----------------
    def _need_grid(self):
        if self.nlat == 0:
            raise RuntimeError("Grid not set. Call .set_grid() method.")

    def _batch(self, nf):
        if self._lib.shtns_set_batch(self._cfg, int(nf), int(self.nlm), int(self.nspat)) != 0:
            capi.check(self._lib)

    def _stream(self):
        s = torch.cuda.current_stream().cuda_stream
        self._lib.cushtns_set_streams(self._cfg, C.c_void_p(s), None)

    # ---------------- transforms ----------------
    def synth(self, *arg, ltr=None):
        """v = synth(qlm); vt, vp = synth(slm, tlm); vr, vt, vp = synth(qlm, slm, tlm)
        (shtns_numpy.i:396-425).  With ltr, the truncated _l transform."""
        self._need_grid()
        n = len(arg)
        if n < 1 or n > 3:
            raise RuntimeError("1,2 or 3 arguments required.")
        ltr = self.lmax if ltr is None else int(ltr)
        if _is_torch(arg[0]):
            return self._synth_torch(arg, ltr)
        q = []
        for a in arg:
            a = np.asarray(a)
            if a.shape[-1] != self.nlm:
                raise RuntimeError("spectral array has wrong size.")
            if a.dtype != np.complex128:
                raise RuntimeError("spectral array should be dtype=complex.")
            q.append(np.ascontiguousarray(a))
        lead = q[0].shape[:-1]
        nf = int(np.prod(lead)) if lead else 1
        outs = [np.empty(lead + self.spat_shape) for _ in range(n)]
        self._batch(nf)
        P = [x.ctypes.data_as(C.c_void_p) for x in q]
        O = [x.ctypes.data_as(C.c_void_p) for x in outs]
        L = self._lib
        if n == 1:
            L.SH_to_spat_l(self._cfg, P[0], O[0], ltr)
        elif n == 2:
            L.SHsphtor_to_spat_l(self._cfg, P[0], P[1], O[0], O[1], ltr)
        else:
            L.SHqst_to_spat_l(self._cfg, P[0], P[1], P[2], O[0], O[1], O[2], ltr)
        capi.check(L)
        return outs[0] if n == 1 else tuple(outs)

    def analys(self, *arg, ltr=None):
        """qlm = analys(v); slm, tlm = analys(vt, vp); qlm, slm, tlm = analys(vr, vt, vp)
        (shtns_numpy.i:427-456).  Inputs are left unchanged."""
        self._need_grid()
        n = len(arg)
        if n < 1 or n > 3:
            raise RuntimeError("1,2 or 3 arguments required.")
        ltr = self.lmax if ltr is None else int(ltr)
        if _is_torch(arg[0]):
            return self._analys_torch(arg, ltr)
        v = []
        for a in arg:
            a = np.asarray(a)
            if a.shape[-2:] != self.spat_shape:
                raise RuntimeError("spatial array has wrong shape.")
            if a.dtype != np.float64:
                raise RuntimeError("spatial array should be dtype=float64.")
            v.append(np.ascontiguousarray(a))
        lead = v[0].shape[:-2]
        nf = int(np.prod(lead)) if lead else 1
        outs = [np.empty(lead + (self.nlm,), dtype=np.complex128) for _ in range(n)]
        self._batch(nf)
        P = [x.ctypes.data_as(C.c_void_p) for x in v]
        O = [x.ctypes.data_as(C.c_void_p) for x in outs]
        L = self._lib
        if n == 1:
            L.spat_to_SH_l(self._cfg, P[0], O[0], ltr)
        elif n == 2:
            L.spat_to_SHsphtor_l(self._cfg, P[0], P[1], O[0], O[1], ltr)
        else:
            L.spat_to_SHqst_l(self._cfg, P[0], P[1], P[2], O[0], O[1], O[2], ltr)
        capi.check(L)
        return outs[0] if n == 1 else tuple(outs)

    def synth_grad(self, slm):
        """(vtheta, vphi) = gradient of slm (SHsph_to_spat)."""
        self._need_grid()
        z = np.zeros_like(slm)
        return self.synth(slm, z)

    # ---------------- torch (device) path ----------------
    def _synth_torch(self, arg, ltr):
        q = []
        for a in arg:
            if not a.is_cuda or a.dtype != torch.complex128 or a.shape[-1] != self.nlm:
                raise RuntimeError("spectral tensors must be CUDA complex128 with last dimension nlm")
            q.append(a.contiguous())
        lead = tuple(q[0].shape[:-1])
        nf = int(np.prod(lead)) if lead else 1
        outs = [torch.empty(lead + self.spat_shape, dtype=torch.float64, device=q[0].device) for _ in q]
        self.synth_into(q, outs, ltr)
        return outs[0] if len(outs) == 1 else tuple(outs)

    def _analys_torch(self, arg, ltr):
        v = []
        for a in arg:
            if not a.is_cuda or a.dtype != torch.float64 or tuple(a.shape[-2:]) != self.spat_shape:
                raise RuntimeError("spatial tensors must be CUDA float64 with trailing shape spat_shape")
            v.append(a.contiguous())
        lead = tuple(v[0].shape[:-2])
        outs = [torch.empty(lead + (self.nlm,), dtype=torch.complex128, device=v[0].device) for _ in v]
        self.analys_into(v, outs, ltr)
        return outs[0] if len(outs) == 1 else tuple(outs)

    def synth_into(self, q, outs, ltr=None):
        """Device synthesis into preallocated tensors (no allocation by torch):
        q: list of 1-3 complex128 CUDA tensors (..., nlm); outs: float64 (..., *spat_shape)."""
        ltr = self.lmax if ltr is None else int(ltr)
        nf = q[0].numel() // self.nlm
        self._batch(nf)
        self._stream()
        P = [C.c_void_p(x.data_ptr()) for x in q]
        O = [C.c_void_p(x.data_ptr()) for x in outs]
        L = self._lib
        if len(q) == 1:
            L.cu_SH_to_spat(self._cfg, P[0], O[0], ltr)
        elif len(q) == 2:
            L.cu_SHsphtor_to_spat(self._cfg, P[0], P[1], O[0], O[1], ltr)
        else:
            L.cu_SHqst_to_spat(self._cfg, P[0], P[1], P[2], O[0], O[1], O[2], ltr)
        capi.check(L)

    def analys_into(self, v, outs, ltr=None):
        """Device analysis into preallocated tensors (see synth_into)."""
        ltr = self.lmax if ltr is None else int(ltr)
        nf = v[0].numel() // self.nspat
        self._batch(nf)
        self._stream()
        P = [C.c_void_p(x.data_ptr()) for x in v]
        O = [C.c_void_p(x.data_ptr()) for x in outs]
        L = self._lib
        if len(v) == 1:
            L.cu_spat_to_SH(self._cfg, P[0], O[0], ltr)
        elif len(v) == 2:
            L.cu_spat_to_SHsphtor(self._cfg, P[0], P[1], O[0], O[1], ltr)
        else:
            L.cu_spat_to_SHqst(self._cfg, P[0], P[1], P[2], O[0], O[1], O[2], ltr)
        capi.check(L)

    # ---------------- fixed order, no FFT (shtns_numpy.i:661-704) ----------------
    def _ml_check(self, im, spec, spat):
        self._need_grid()
        nel = self.lmax + 1 - abs(int(im)) * self.mres
        for a in spec:
            if a.dtype != np.complex128 or a.size != nel or not a.flags.c_contiguous:
                raise RuntimeError("spectral array of an order must be contiguous complex128 of size %d" % nel)
        for a in spat:
            if a.dtype != np.complex128 or a.size != self.nlat or not a.flags.c_contiguous:
                raise RuntimeError("spatial array of an order must be contiguous complex128 of size nlat")

    def _ml(self, fn, im, *arrays):
        P = [a.ctypes.data_as(C.c_void_p) for a in arrays]
        getattr(self._lib, fn)(self._cfg, int(im), *P, int(self.lmax))
        capi.check(self._lib)

    def spat_to_SH_m(self, Vr, Qlm, im):
        self._ml_check(im, [Qlm], [Vr]); self._ml("spat_to_SH_ml", im, Vr, Qlm)

    def SH_to_spat_m(self, Qlm, Vr, im):
        self._ml_check(im, [Qlm], [Vr]); self._ml("SH_to_spat_ml", im, Qlm, Vr)

    def spat_to_SHsphtor_m(self, Vt, Vp, Slm, Tlm, im):
        self._ml_check(im, [Slm, Tlm], [Vt, Vp]); self._ml("spat_to_SHsphtor_ml", im, Vt, Vp, Slm, Tlm)

    def SHsphtor_to_spat_m(self, Slm, Tlm, Vt, Vp, im):
        self._ml_check(im, [Slm, Tlm], [Vt, Vp]); self._ml("SHsphtor_to_spat_ml", im, Slm, Tlm, Vt, Vp)

    def SHsph_to_spat_m(self, Slm, Vt, Vp, im):
        self._ml_check(im, [Slm], [Vt, Vp]); self._ml("SHsph_to_spat_ml", im, Slm, Vt, Vp)

    def SHtor_to_spat_m(self, Tlm, Vt, Vp, im):
        self._ml_check(im, [Tlm], [Vt, Vp]); self._ml("SHtor_to_spat_ml", im, Tlm, Vt, Vp)

    def spat_to_SHqst_m(self, Vr, Vt, Vp, Qlm, Slm, Tlm, im):
        self._ml_check(im, [Qlm, Slm, Tlm], [Vr, Vt, Vp]); self._ml("spat_to_SHqst_ml", im, Vr, Vt, Vp, Qlm, Slm, Tlm)

    def SHqst_to_spat_m(self, Qlm, Slm, Tlm, Vr, Vt, Vp, im):
        self._ml_check(im, [Qlm, Slm, Tlm], [Vr, Vt, Vp]); self._ml("SHqst_to_spat_ml", im, Qlm, Slm, Tlm, Vr, Vt, Vp)

    # ---------------- complex-valued fields (shtns_numpy.i:469-545) ----------------
    def zidx(self, l, m):
        """index l(l+1)+m of (l, m) in a complex-field expansion (lmax = mmax)"""
        l = np.asarray(l)
        m = np.asarray(m)
        return l * (l + 1) + m

    def _cplx_ready(self):
        self._need_grid()
        if self.lmax != self.mmax or self.mres != 1:
            raise RuntimeError("complex SH requires lmax=mmax and mres=1.")

    def synth_cplx(self, *arg):
        """z = synth_cplx(zlm); zt, zp = synth_cplx(slm, tlm); zr, zt, zp =
        synth_cplx(qlm, slm, tlm): complex-valued spatial fields from
        (lmax+1)^2 complex coefficients each."""
        self._cplx_ready()
        n = len(arg)
        if n < 1 or n > 3:
            raise RuntimeError("1,2 or 3 arguments required.")
        q = []
        for a in arg:
            a = np.ascontiguousarray(a)
            if a.size != (self.lmax + 1) ** 2:
                raise RuntimeError("spectral array has wrong size.")
            if a.dtype != np.complex128:
                raise RuntimeError("spectral array should be dtype=complex.")
            q.append(a)
        outs = [np.empty(self.spat_shape, dtype=np.complex128) for _ in range(n)]
        fn = {1: "SH_to_spat_cplx", 2: "SHsphtor_to_spat_cplx", 3: "SHqst_to_spat_cplx"}[n]
        getattr(self._lib, fn)(self._cfg, *[x.ctypes.data_as(C.c_void_p) for x in q + outs])
        capi.check(self._lib)
        return outs[0] if n == 1 else tuple(outs)

    def analys_cplx(self, *arg):
        """zlm = analys_cplx(z); slm, tlm = analys_cplx(zt, zp); qlm, slm, tlm =
        analys_cplx(zr, zt, zp)."""
        self._cplx_ready()
        n = len(arg)
        if n < 1 or n > 3:
            raise RuntimeError("1,2 or 3 arguments required.")
        v = []
        for a in arg:
            a = np.ascontiguousarray(a)
            if a.shape != self.spat_shape:
                raise RuntimeError("spatial array has wrong shape.")
            if a.dtype != np.complex128:
                raise RuntimeError("spatial array should be dtype=complex128.")
            v.append(a)
        outs = [np.empty((self.lmax + 1) ** 2, dtype=np.complex128) for _ in range(n)]
        fn = {1: "spat_cplx_to_SH", 2: "spat_cplx_to_SHsphtor", 3: "spat_cplx_to_SHqst"}[n]
        getattr(self._lib, fn)(self._cfg, *[x.ctypes.data_as(C.c_void_p) for x in v + outs])
        capi.check(self._lib)
        return outs[0] if n == 1 else tuple(outs)

    # ---------------- local evaluation (shtns_numpy.i:566-606) ----------------
    def _spec(self, a, n=None):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        if a.size != (self.nlm if n is None else n):
            raise RuntimeError("spectral array has wrong size.")
        return a

    def SH_to_point(self, Qlm, cost, phi):
        """Value of the real scalar field Qlm at cos(theta) = cost, longitude phi."""
        q = self._spec(Qlm)
        v = self._lib.SH_to_point(self._cfg, q.ctypes.data_as(C.c_void_p), float(cost), float(phi))
        capi.check(self._lib)
        return v

    def SH_to_point_cplx(self, alm, cost, phi):
        """Value of the complex field alm (LM_cplx layout) at (cost, phi)."""
        a = self._spec(alm, (self.lmax + 1) ** 2)
        z = self._lib.SH_to_point_cplx(self._cfg, a.ctypes.data_as(C.c_void_p), float(cost), float(phi))
        capi.check(self._lib)
        return complex(z.re, z.im)

    def _point3(self, fn, arrs, cost, phi):
        out = [C.c_double() for _ in range(3)]
        getattr(self._lib, fn)(self._cfg, *[a.ctypes.data_as(C.c_void_p) for a in arrs], float(cost), float(phi),
                               *[C.byref(o) for o in out])
        capi.check(self._lib)
        return tuple(o.value for o in out)

    def SH_to_grad_point(self, DrSlm, Slm, cost, phi):
        """(vr, vt, vp): vr from DrSlm, (vt, vp) the gradient of Slm."""
        return self._point3("SH_to_grad_point", [self._spec(DrSlm), self._spec(Slm)], cost, phi)

    def SHqst_to_point(self, Qlm, Slm, Tlm, cost, phi):
        """(vr, vt, vp) of the vector field (Qlm, Slm, Tlm) at (cost, phi)."""
        return self._point3("SHqst_to_point", [self._spec(Qlm), self._spec(Slm), self._spec(Tlm)], cost, phi)

    def SH_to_lat(self, Qlm, cost, Vr, ltr=None, mtr=None):
        """Fill Vr (nphi doubles) with the field on latitude cost at phi_j = 2 pi j / nphi."""
        q = self._spec(Qlm)
        if Vr.dtype != np.float64 or not Vr.flags.c_contiguous:
            raise RuntimeError("Vr must be a contiguous float64 array.")
        self._lib.SH_to_lat(self._cfg, q.ctypes.data_as(C.c_void_p), float(cost), Vr.ctypes.data_as(C.c_void_p),
                            int(Vr.size), self.lmax if ltr is None else int(ltr), self.mmax if mtr is None else int(mtr))
        capi.check(self._lib)

    def SHqst_to_lat(self, Qlm, Slm, Tlm, cost, Vr, Vt, Vp, ltr=None, mtr=None):
        n = Vr.size
        for v in (Vr, Vt, Vp):
            if v.dtype != np.float64 or not v.flags.c_contiguous or v.size != n:
                raise RuntimeError("Vr, Vt, Vp must be contiguous float64 arrays of one size.")
        arrs = [self._spec(a) for a in (Qlm, Slm, Tlm)]
        self._lib.SHqst_to_lat(self._cfg, *[a.ctypes.data_as(C.c_void_p) for a in arrs], float(cost),
                               *[v.ctypes.data_as(C.c_void_p) for v in (Vr, Vt, Vp)], int(n),
                               self.lmax if ltr is None else int(ltr), self.mmax if mtr is None else int(mtr))
        capi.check(self._lib)

    def points(self, Qlm, cost, phi):
        """Values of the scalar field Qlm (CUDA complex128, nlm) at the points
        (cost[i], phi[i]) (CUDA float64 tensors), one CUDA launch."""
        if not (_is_torch(Qlm) and Qlm.is_cuda):
            raise RuntimeError("points() takes CUDA tensors")
        q = Qlm.contiguous()
        ct, ph = cost.contiguous().double(), phi.contiguous().double()
        v = torch.empty_like(ct)
        self._stream()
        self._lib.shtns_b200_SH_to_points(self._cfg, C.c_void_p(q.data_ptr()), C.c_void_p(ct.data_ptr()),
                                          C.c_void_p(ph.data_ptr()), C.c_void_p(v.data_ptr()), int(ct.numel()))
        capi.check(self._lib)
        return v

    def mul_ct_matrix(self):
        mx = np.zeros(2 * self.nlm)
        self._lib.mul_ct_matrix(self._cfg, mx.ctypes.data_as(C.c_void_p))
        return mx

    def st_dt_matrix(self):
        mx = np.zeros(2 * self.nlm)
        self._lib.st_dt_matrix(self._cfg, mx.ctypes.data_as(C.c_void_p))
        return mx

    def SH_mul_mx(self, mx, Qlm):
        m = np.ascontiguousarray(mx, dtype=np.float64)
        if m.size != 2 * self.nlm:
            raise RuntimeError("matrix has wrong size.")
        q = self._spec(Qlm)
        r = np.empty_like(q)
        self._lib.SH_mul_mx(self._cfg, m.ctypes.data_as(C.c_void_p), q.ctypes.data_as(C.c_void_p),
                            r.ctypes.data_as(C.c_void_p))
        capi.check(self._lib)
        return r

    # ---------------- rotations (shtns_numpy.i:608-649) ----------------
    def _rot(self, fn, Qlm, *args):
        q = self._spec(Qlm)
        r = np.empty_like(q)
        getattr(self._lib, fn)(self._cfg, q.ctypes.data_as(C.c_void_p), *args, r.ctypes.data_as(C.c_void_p))
        capi.check(self._lib)
        return r

    def Zrotate(self, Qlm, alpha):
        """Rotation about the z axis by alpha (Rlm = Qlm e^{-i m alpha})."""
        return self._rot("SH_Zrotate", Qlm, float(alpha))

    def Yrotate(self, Qlm, alpha):
        """Rotation about the y axis by alpha (mres = 1, mmax = lmax)."""
        return self._rot("SH_Yrotate", Qlm, float(alpha))

    def Yrotate90(self, Qlm):
        return self._rot("SH_Yrotate90", Qlm)

    def Xrotate90(self, Qlm):
        return self._rot("SH_Xrotate90", Qlm)


class rotation:
    """Rotation of spherical-harmonic expansions (shtns_numpy.i:717-771):
    rotation(lmax, mmax=-1, norm=0), then set_angles_ZYZ / set_angles_ZXZ /
    set_angle_axis and apply_real / apply_cplx (orthonormal expansions of
    real fields, LM layout, or complex fields, LM_cplx layout)."""

    def __init__(self, lmax, mmax=-1, norm=0):
        self._lib = capi.load()
        if mmax < 0:
            mmax = lmax
        self._r = self._lib.shtns_rotation_create(int(lmax), int(mmax), int(norm))
        if not self._r:
            raise SHTError(self._lib.shtns_b200_last_error().decode())
        self.lmax, self.mmax = lmax, mmax
        self.nlm = int(self._lib.nlm_calc(lmax, mmax, 1))
        self.nlm_cplx = int(self._lib.nlm_cplx_calc(lmax, mmax, 1))

    def __del__(self):
        try:
            if getattr(self, "_r", None):
                self._lib.shtns_rotation_destroy(self._r)
                self._r = None
        except Exception:
            pass

    def set_angles_ZYZ(self, alpha, beta, gamma):
        self._lib.shtns_rotation_set_angles_ZYZ(self._r, float(alpha), float(beta), float(gamma))
        capi.check(self._lib)

    def set_angles_ZXZ(self, alpha, beta, gamma):
        self._lib.shtns_rotation_set_angles_ZXZ(self._r, float(alpha), float(beta), float(gamma))
        capi.check(self._lib)

    def set_angle_axis(self, theta, Vx, Vy, Vz):
        self._lib.shtns_rotation_set_angle_axis(self._r, float(theta), float(Vx), float(Vy), float(Vz))
        capi.check(self._lib)

    def wigner_d_matrix(self, l):
        """(2l+1, 2l+1) Wigner d-matrix of the y rotation by beta, entry [m'+l, m+l]."""
        mx = np.zeros((2 * l + 1, 2 * l + 1))
        n = self._lib.shtns_rotation_wigner_d_matrix(self._r, int(l), mx.ctypes.data_as(C.c_void_p))
        capi.check(self._lib)
        if n == 0:
            raise ValueError("0 <= l <= lmax not satisfied")
        return mx

    def _apply(self, fn, a, n):
        q = np.ascontiguousarray(a, dtype=np.complex128)
        if q.size != n:
            raise RuntimeError("spectral array has wrong size.")
        r = np.empty_like(q)
        getattr(self._lib, fn)(self._r, q.ctypes.data_as(C.c_void_p), r.ctypes.data_as(C.c_void_p))
        capi.check(self._lib)
        return r

    def apply_real(self, Qlm):
        return self._apply("shtns_rotation_apply_real", Qlm, self.nlm)

    def apply_cplx(self, Zlm):
        return self._apply("shtns_rotation_apply_cplx", Zlm, self.nlm_cplx)


def _inplace(fn, kinds):
    """Method writing into caller arrays, as the reference's in-place
    transforms (shtns_numpy.i:319-395): one field, sizes checked."""
    def method(self, *arrs):
        self._need_grid()
        if len(arrs) != len(kinds):
            raise RuntimeError("%d arrays required." % len(kinds))
        sizes = {"q": (np.complex128, self.nlm), "v": (np.float64, self.nspat),
                 "a": (np.complex128, (self.lmax + 1) ** 2), "z": (np.complex128, self.nspat)}
        ptrs = []
        for a, k in zip(arrs, kinds):
            dt, n = sizes[k]
            if not isinstance(a, np.ndarray) or not a.flags.c_contiguous or a.dtype != dt or a.size != n:
                raise RuntimeError("array must be a contiguous %s array of %d elements." % (np.dtype(dt).name, n))
            ptrs.append(a.ctypes.data_as(C.c_void_p))
        self._batch(1)
        getattr(self._lib, fn)(self._cfg, *ptrs)
        capi.check(self._lib)
    method.__name__ = fn
    method.__doc__ = "%s(%s) in place (shtns_numpy.i:319-395)." % (fn, ", ".join(kinds))
    return method


for _fn, _k in (("spat_to_SH", "vq"), ("SH_to_spat", "qv"), ("spat_cplx_to_SH", "za"), ("SH_to_spat_cplx", "az"),
                ("spat_to_SHsphtor", "vvqq"), ("SHsphtor_to_spat", "qqvv"), ("SHsph_to_spat", "qvv"),
                ("SHtor_to_spat", "qvv"), ("spat_cplx_to_SHsphtor", "zzaa"), ("SHsphtor_to_spat_cplx", "aazz"),
                ("spat_to_SHqst", "vvvqqq"), ("SHqst_to_spat", "qqqvvv"), ("spat_cplx_to_SHqst", "zzzaaa"),
                ("SHqst_to_spat_cplx", "aaazzz")):
    setattr(sht, _fn, _inplace(_fn, _k))


def _zlm(self, idx):
    """(l, m) of index idx in the complex expansion (shtns_numpy.i:545-553)."""
    idx = np.asarray(idx)
    if (idx >= (self.lmax + 1) ** 2).any() or (idx < 0).any():
        raise RuntimeError("invalid range for l,m")
    l = np.sqrt(idx).astype(int)
    return l, idx - l * (l + 1)


def _spec_array_cplx(self):
    return np.zeros((self.lmax + 1) ** 2, dtype=complex)


def _spat_array_cplx(self):
    if self.nlat == 0:
        raise RuntimeError("Grid not set. Call .set_grid() method.")
    return np.zeros(self.spat_shape, dtype="complex128")


sht.zlm = _zlm
sht.spec_array_cplx = _spec_array_cplx
sht.spat_array_cplx = _spat_array_cplx
