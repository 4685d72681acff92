"""cuFFT through ctypes with the reference's plan for theta-contiguous grids
(sht_gpu.cu:186-190): a Z2Z transform of length nphi over the nlat/2
latitude pairs of one field (adjacent latitudes as real and imaginary parts),
istride = ostride = nlat/2, idist = odist = 1.

Test and measurement infrastructure only: the cross-check of the library's
own FFT kernels and the timing beside them.  The library never calls cuFFT."""
import ctypes as C
import os

CUFFT_Z2Z = 0x69
CUFFT_FORWARD = -1
CUFFT_INVERSE = 1

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    cands = []
    try:
        import nvidia.cufft
        cands.append(os.path.join(list(nvidia.cufft.__path__)[0], "lib", "libcufft.so.11"))
    except ImportError:
        pass
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cands += [os.path.join(cuda, "lib64", "libcufft.so.11"), "libcufft.so.11"]
    err = None
    for c in cands:
        try:
            L = C.CDLL(c)
            break
        except OSError as e:
            err = e
    else:
        raise OSError(f"libcufft not found: {err}")
    L.cufftPlanMany.argtypes = [C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_int,
                                C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int, C.c_int]
    L.cufftSetStream.argtypes = [C.c_int, C.c_void_p]
    L.cufftExecZ2Z.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    L.cufftDestroy.argtypes = [C.c_int]
    _lib = L
    return L


class PairPlan:
    """The reference's theta-contiguous cuFFT plan for one field."""

    def __init__(self, nphi, nlat, stream=None):
        L = lib()
        self.h = C.c_int(0)
        n = (C.c_int * 1)(nphi)
        p = nlat // 2
        r = L.cufftPlanMany(C.byref(self.h), 1, n, n, p, 1, n, p, 1, CUFFT_Z2Z, p)
        if r != 0:
            raise RuntimeError(f"cufftPlanMany failed ({r})")
        if stream is not None:
            L.cufftSetStream(self.h, C.c_void_p(stream))

    def exec(self, src, dst, direction):
        r = lib().cufftExecZ2Z(self.h, C.c_void_p(src), C.c_void_p(dst), direction)
        if r != 0:
            raise RuntimeError(f"cufftExecZ2Z failed ({r})")

    def destroy(self):
        lib().cufftDestroy(self.h)
