"""fg_kinetic_energy_dipo_noalloc (allocation-free, static device scratch)
against fg_kinetic_energy_dipo of a context holding the same momenta."""
import ctypes as C

import numpy as np
import pytest

import helpers
from feram_b200 import _capi as A


def _layer_tables(p):
    """Per-layer m^-1 and sum_p mask as alloc_Coord / read_defects_u.F:52-69
    set them: film and epit count the lower (Lz+1)/2 layers, gap layers
    have no mass and are not counted."""
    minv = np.full(p.Lz, 1.0 / p.mass_dipo[0])
    mask = np.ones(p.Lz, dtype=np.uint8)
    if p.bulk_or_film in (A.FG_FILM, A.FG_EPIT):
        mask[(p.Lz + 1) // 2:] = 0
    if p.gap_id > 0:
        minv[0], mask[0] = 0.0, 0
        if p.gap_id == 2:
            minv[p.Lz // 2], mask[p.Lz // 2] = 0.0, 0
    return minv, mask


def _call(dev_p, p, minv, mask, stream, ke_ptr):
    err = C.create_string_buffer(256)
    rc = A.lib().fg_kinetic_energy_dipo_noalloc(
        C.c_void_p(dev_p), p.Lx, p.Ly, p.Lz, minv.ctypes.data_as(C.POINTER(C.c_double)),
        mask.ctypes.data_as(C.POINTER(C.c_ubyte)), C.c_void_p(stream), C.c_void_p(ke_ptr), err, 256)
    return rc, err.value.decode()


@pytest.mark.gpu
@pytest.mark.parametrize("case", [dict(L="16 16 16"), dict(L="12 10 8", bulk_or_film="'film'")],
                         ids=["bulk16", "film12x10x8"])
def test_noalloc_matches_context(fg, case):
    import torch
    p = helpers.params(kelvin="300", **case)
    u = helpers.seeded_u(p, 41, sigma=0.05)
    q = helpers.seeded_p(p, 42, sigma=0.01)
    with fg.Context(p, A.FG_PREC_FP64) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        ke_ref = ctx.kinetic_energy_dipo()
    soa = np.ascontiguousarray(np.moveaxis(A.physical(q, p), -1, 0))  # [3][z][y][x]
    dev_p = torch.from_numpy(soa).to("cuda")
    ke = torch.zeros(2, dtype=torch.float64, device="cuda")
    minv, mask = _layer_tables(p)
    stream = torch.cuda.current_stream().cuda_stream
    for k in range(2):  # two calls in a row share the static scratch
        rc, msg = _call(dev_p.data_ptr(), p, minv, mask, stream, ke.data_ptr() + 8 * k)
        assert rc == A.FG_OK, msg
    torch.cuda.synchronize()
    got = ke.cpu().numpy()
    assert np.all(np.abs(got - ke_ref) <= 1e-12 * abs(ke_ref)), (got, ke_ref)


def test_noalloc_rejects_oversized_and_bad_input(fg):
    """Argument checks run on the host before any device work."""
    p = helpers.params(L="8 8 8")
    minv, mask = _layer_tables(p)
    big = A.fg_params.from_buffer_copy(p)
    big.Lz = 1025
    minv_big = np.ones(big.Lz)
    mask_big = np.ones(big.Lz, dtype=np.uint8)
    rc, msg = _call(16, big, minv_big, mask_big, 0, 16)
    assert rc == A.FG_ERR_ARG and "FG_NOALLOC_MAX_LZ" in msg, (rc, msg)
    rc, msg = _call(16, p, minv, np.zeros_like(mask), 0, 16)
    assert rc == A.FG_ERR_ARG and "no layer" in msg, (rc, msg)
    rc, msg = _call(0, p, minv, mask, 0, 16)
    assert rc == A.FG_ERR_ARG and "null" in msg, (rc, msg)
