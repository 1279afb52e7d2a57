"""cuFFT through ctypes, as the reference's cufft_check.F:180-207 calls it:
cufftPlanMany of rank 3 over (Lz, Ly, Lx) with the padded embeds
(Lz, Ly+padding_y, 2(Lx/2+1)) and (Lz, Ly+padding_y, Lx/2+1), stride =
howmany, dist = 1 (the interleaved component layout of coord_module.F:91-93),
D2Z / Z2D (and R2C / C2R for FP32).

Test and measurement infrastructure only: cuFFT is the cross-check and the
speed bar of the device FFT, never part of the product path.  Device memory
comes from torch (its tensors' data pointers); cuFFT runs on the legacy
default stream, which is torch's current stream unless changed.
"""
import ctypes as C
import glob
import os

CUFFT_R2C, CUFFT_C2R, CUFFT_D2Z, CUFFT_Z2D = 0x2A, 0x2C, 0x6A, 0x6C
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    import torch
    cands = glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cufft", "lib", "libcufft.so*"))
    cands += ["/usr/local/cuda/lib64/libcufft.so"]
    err = None
    for c in cands:
        try:
            L = C.CDLL(c)
            break
        except OSError as e:
            err = e
    else:
        raise OSError(f"cuFFT not found: {err}")
    ip = C.POINTER(C.c_int)
    L.cufftPlanMany.argtypes = [ip, C.c_int, ip, ip, C.c_int, C.c_int, ip, C.c_int, C.c_int, C.c_int, C.c_int]
    L.cufftPlanMany.restype = C.c_int
    for n in ("cufftExecD2Z", "cufftExecZ2D", "cufftExecR2C", "cufftExecC2R"):
        f = getattr(L, n)
        f.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        f.restype = C.c_int
    L.cufftDestroy.argtypes = [C.c_int]
    L.cufftDestroy.restype = C.c_int
    _lib = L
    return L


class PlanMany:
    """Forward (real -> half complex) and backward plans of cufft_check.F on
    the padded interleaved layout; fp64 selects D2Z/Z2D, else R2C/C2R."""

    def __init__(self, Lx, Ly, Lz, padding_y=1, howmany=3, fp64=True, layout="reference"):
        L = load()
        n = (C.c_int * 3)(Lz, Ly, Lx)
        self.fp64 = fp64
        self.fwd, self.bwd = C.c_int(), C.c_int()
        if layout == "reference":  # interleaved components, padded embeds
            a = (C.c_int * 3)(Lz, Ly + padding_y, 2 * (Lx // 2 + 1))
            w = (C.c_int * 3)(Lz, Ly + padding_y, Lx // 2 + 1)
            args_f = (a, howmany, 1, w, howmany, 1)
            args_b = (w, howmany, 1, a, howmany, 1)
        else:  # "contiguous": one unpadded field after the other
            nr, nc = Lx * Ly * Lz, (Lx // 2 + 1) * Ly * Lz
            args_f = (None, 1, nr, None, 1, nc)
            args_b = (None, 1, nc, None, 1, nr)
        tf, tb = (CUFFT_D2Z, CUFFT_Z2D) if fp64 else (CUFFT_R2C, CUFFT_C2R)
        rc = L.cufftPlanMany(C.byref(self.fwd), 3, n, *args_f, tf, howmany)
        rc2 = L.cufftPlanMany(C.byref(self.bwd), 3, n, *args_b, tb, howmany)
        if rc or rc2:
            raise RuntimeError(f"cufftPlanMany failed: {rc}, {rc2}")

    def forward(self, real_ptr, cplx_ptr):
        f = load().cufftExecD2Z if self.fp64 else load().cufftExecR2C
        rc = f(self.fwd.value, C.c_void_p(real_ptr), C.c_void_p(cplx_ptr))
        if rc:
            raise RuntimeError(f"cufft forward: {rc}")

    def backward(self, cplx_ptr, real_ptr):
        f = load().cufftExecZ2D if self.fp64 else load().cufftExecC2R
        rc = f(self.bwd.value, C.c_void_p(cplx_ptr), C.c_void_p(real_ptr))
        if rc:
            raise RuntimeError(f"cufft backward: {rc}")

    def close(self):
        L = load()
        for h in (self.fwd, self.bwd):
            if h.value:
                L.cufftDestroy(h.value)
                h.value = 0
