"""The device FFT against cuFFT on the same B200: the batched 3-component
r2c and c2r of fg_fft_r2c3 / fg_fft_c2r3 against cuFFT D2Z / Z2D (FP64) and
R2C / C2R (FP32) planned as the reference's cufft_check.F:180-207 plans them
(rank 3, padded embeds, stride = howmany = 3, dist = 1).  cuFFT is the
cross-check only; nothing in the product links it."""
import numpy as np
import pytest

import cufft_lib
import helpers
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu

TOL = {A.FG_PREC_FP64: 2e-13, A.FG_PREC_MIXED: 3e-6}
SHAPES = [(32, 32, 32), (128, 128, 128), (20, 12, 18)]


def _cufft_roundtrip(f, p, fp64):
    """cuFFT forward of the padded real field f, then backward of that
    spectrum (unnormalised), as numpy arrays in the reference layouts."""
    import torch
    dt, ct = (torch.float64, torch.complex128) if fp64 else (torch.float32, torch.complex64)
    x = torch.from_numpy(f).to("cuda", dt).contiguous()
    X = torch.zeros(A.complex_field(p).shape, dtype=ct, device="cuda")
    y = torch.zeros_like(x)
    plan = cufft_lib.PlanMany(p.Lx, p.Ly, p.Lz, p.padding_y, 3, fp64)
    try:
        plan.forward(x.data_ptr(), X.data_ptr())
        Xc = X.clone()  # c2r may overwrite its input
        plan.backward(Xc.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
    finally:
        plan.close()
    return X.cpu().numpy().astype(np.complex128), y.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_device_fft_matches_cufft(fg, shape, prec):
    Lx, Ly, Lz = shape
    p = helpers.params(L=f"{Lx} {Ly} {Lz}")
    rng = np.random.default_rng(Lx * 10000 + Ly * 100 + Lz)
    f = A.real_field(p)
    A.physical(f, p)[...] = rng.standard_normal((Lz, Ly, Lx, 3))
    if prec == A.FG_PREC_MIXED:
        f = f.astype(np.float32).astype(np.float64)
    Xc, yc = _cufft_roundtrip(f, p, prec == A.FG_PREC_FP64)
    with fg.Context(p, prec) as ctx:
        X = ctx.fft_r2c3(f)
        y = ctx.fft_c2r3(Xc)  # the same spectrum into both inverses
    s = np.abs(Xc[:, :Ly]).max()
    err_f = np.abs(X[:, :Ly] - Xc[:, :Ly]).max() / s
    r = np.abs(A.physical(yc, p)).max()
    err_b = np.abs(A.physical(y, p) - A.physical(yc, p)).max() / r
    assert err_f <= TOL[prec], err_f
    assert err_b <= TOL[prec] * 5, err_b


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_time_fft_reports_positive_times(fg, prec):
    p = helpers.params(L="32 32 32")
    with fg.Context(p, prec) as ctx:
        ms = ctx.time_fft(5)
    assert ms[0] > 0 and ms[1] > 0 and ms[0] < 100 and ms[1] < 100, ms
