"""Device FFT and k-space tables against numpy and the oracle (C-ABI calls)."""
import numpy as np
import pytest

import helpers
import oracle_lib
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu

# (24, 24, 24), (48, 48, 48): the compile-time transforms with a radix-3 stage
SHAPES = [(16, 16, 16), (12, 10, 6), (20, 12, 18), (8, 15, 9), (32, 24, 20), (24, 24, 24), (48, 48, 48)]
TOL = {A.FG_PREC_FP64: 2e-13, A.FG_PREC_MIXED: 2e-6}


def _ctx(fg, shape, prec, **tags):
    p = helpers.params(L="%d %d %d" % shape, **tags)
    return p, fg.Context(p, prec)


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
@pytest.mark.parametrize("shape", SHAPES)
def test_fft_r2c3_matches_numpy(fg, shape, prec):
    p, ctx = _ctx(fg, shape, prec)
    rng = np.random.default_rng(11)
    f = A.real_field(p)
    A.physical(f, p)[...] = rng.standard_normal((p.Lz, p.Ly, p.Lx, 3))
    out = ctx.fft_r2c3(f)
    ref = np.fft.rfftn(A.physical(f, p), axes=(0, 1, 2))
    err = np.abs(out[:, :p.Ly] - ref).max() / np.abs(ref).max()
    assert err <= TOL[prec], err
    ctx.close()


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
@pytest.mark.parametrize("shape", SHAPES)
def test_fft_c2r3_matches_numpy_nonhermitian(fg, shape, prec):
    p, ctx = _ctx(fg, shape, prec)
    rng = np.random.default_rng(12)
    X = A.complex_field(p)
    X[:, :p.Ly] = rng.standard_normal(X[:, :p.Ly].shape) + 1j * rng.standard_normal(X[:, :p.Ly].shape)
    back = ctx.fft_c2r3(X)
    ref = np.fft.irfftn(X[:, :p.Ly], s=(p.Lz, p.Ly, p.Lx), axes=(0, 1, 2)) * p.N
    err = np.abs(A.physical(back, p) - ref).max() / np.abs(ref).max()
    assert err <= TOL[prec], err
    assert np.all(back[:, p.Ly:] == 0) and np.all(back[:, :, p.Lx:] == 0)  # padding written as zeros
    ctx.close()


@pytest.mark.parametrize("shape", [(16, 16, 16), (12, 10, 6), (20, 12, 18), (24, 24, 24)])
def test_device_long_range_table_matches_oracle(fg, shape):
    p, ctx = _ctx(fg, shape, A.FG_PREC_FP64)
    ctx.build_tables()
    lr = ctx.get_long_range()
    _, lro = oracle_lib.Oracle(p).tables()
    err = np.abs(lr[:, :p.Ly] - lro[:, :p.Ly]).max() / np.abs(lro).max()
    assert err <= 1e-12, err
    ctx.close()


def test_device_long_range_dispersion_golden(fg):
    g = helpers.golden("dispersion_long64.json")
    p = fg.default_params()
    p.Lx, p.Ly, p.Lz = g["L"]
    p.a0, p.epsilon_inf = g["a0"], g["epsilon_inf"]
    p.Z_star[0] = g["Z_star"]
    p.dt = 0.002
    fg.make_param(p)
    with fg.Context(p, A.FG_PREC_FP64) as ctx:
        ctx.build_tables()
        lr = ctx.get_long_range()
    worst, scale = 0.0, 0.0
    for pt in g["points"]:
        ix, iy, iz = pt["k"]
        M = p.Z_star[0] ** 2 * lr[iz, iy, ix]
        scale = max(scale, np.abs(M).max())
        if (ix, iy, iz) != (0, 0, 0):
            worst = max(worst, np.abs(np.sort(np.linalg.eigvalsh(M)) - np.sort(pt["eig"])).max())
    assert worst <= 1e-12 * scale, worst


def test_upload_rejects_foreign_short_range(fg):
    p, ctx = _ctx(fg, (12, 10, 6), A.FG_PREC_FP64)
    sr, lr = oracle_lib.Oracle(p).tables()
    sr2 = sr.copy()
    sr2[1, 2, 3, 0, 0] += 0.5
    with pytest.raises(fg.FeramError):
        ctx.upload_tables(sr2, lr)
    ctx.upload_tables(sr, lr)
    ctx.close()
