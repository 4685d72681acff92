"""Differentiable scalar transforms for PyTorch.

`synth(sh, q)` and `analys(sh, v)` are torch.autograd.Functions over the
device transforms of a plan `sh` (shtns_b200.sht).  Their backward passes are
the hand-written adjoint kernels of the C ABI (cu_SH_to_spat_adjoint,
cu_spat_to_SH_adjoint): the adjoint of the synthesis is a quadrature-weight-
free analysis scaled by (2 - delta_m0) nphi, the adjoint of the analysis is a
synthesis weighted by the Gauss weight of each latitude.  Gradients of
complex coefficients follow PyTorch's convention dL/dRe + i dL/dIm, so the
real-valued transforms and their adjoints are exact transposes.

Inputs may be complex128/float64 (FP64) or complex64/float32 (FP32: computed
in FP64 on the device and rounded back to FP32).  Leading dimensions batch.
"""
import ctypes as C

import torch

from . import capi


def _call(sh, fn, src, nfields, dst, ltr):
    lib = sh._lib
    sh._batch(nfields)
    sh._stream()
    getattr(lib, fn)(sh._cfg, C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()), int(ltr))
    capi.check(lib)


def _spec64(q):
    return q.to(torch.complex128).contiguous()


def _spat64(v):
    return v.to(torch.float64).contiguous()


class _Synth(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sh, q, ltr):
        ctx.sh, ctx.ltr = sh, ltr
        ctx.in_dtype = q.dtype
        q64 = _spec64(q)
        lead = tuple(q64.shape[:-1])
        nf = q64.numel() // sh.nlm
        v = torch.empty(lead + sh.spat_shape, dtype=torch.float64, device=q.device)
        _call(sh, "cu_SH_to_spat", q64, nf, v, ltr)
        return v if q.dtype == torch.complex128 else v.to(torch.float32)

    @staticmethod
    def backward(ctx, g):
        sh = ctx.sh
        g64 = _spat64(g)
        lead = tuple(g64.shape[:-2])
        nf = g64.numel() // sh.nspat
        qg = torch.empty(lead + (sh.nlm,), dtype=torch.complex128, device=g.device)
        _call(sh, "cu_SH_to_spat_adjoint", g64, nf, qg, ctx.ltr)
        return None, qg.to(ctx.in_dtype), None


class _Analys(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sh, v, ltr):
        ctx.sh, ctx.ltr = sh, ltr
        ctx.in_dtype = v.dtype
        v64 = _spat64(v)
        lead = tuple(v64.shape[:-2])
        nf = v64.numel() // sh.nspat
        q = torch.empty(lead + (sh.nlm,), dtype=torch.complex128, device=v.device)
        _call(sh, "cu_spat_to_SH", v64, nf, q, ltr)
        return q if v.dtype == torch.float64 else q.to(torch.complex64)

    @staticmethod
    def backward(ctx, h):
        sh = ctx.sh
        h64 = _spec64(h)
        lead = tuple(h64.shape[:-1])
        nf = h64.numel() // sh.nlm
        vg = torch.empty(lead + sh.spat_shape, dtype=torch.float64, device=h.device)
        _call(sh, "cu_spat_to_SH_adjoint", h64, nf, vg, ctx.ltr)
        return None, vg.to(ctx.in_dtype), None


def synth(sh, q, ltr=None):
    """Differentiable scalar synthesis: q (..., nlm) complex -> (..., *spat_shape)."""
    return _Synth.apply(sh, q, sh.lmax if ltr is None else int(ltr))


def analys(sh, v, ltr=None):
    """Differentiable scalar analysis: v (..., *spat_shape) real -> (..., nlm)."""
    return _Analys.apply(sh, v, sh.lmax if ltr is None else int(ltr))
