"""Supercell sizes at the edge of what the device path holds.

An x-y plane of (Lx/2 + 1) x Ly complex values is transformed inside one
CTA's shared memory, and the k-space tables are built by FP64 transforms in
both precisions, so the FP64 plane sets the limit: 160 x 160 fits
(81 x 160 x 16 B = 207 KB), 192 x 192 (298 KB) does not.  A plane that does
not fit is refused at fg_create with FG_ERR_UNSUPPORTED (the reference, on
FFTW, has no such limit); the largest one that fits gives the oracle's
force.  Lengths must factor into 2, 3 and 5
(L/2 along x), as the runtime FFT plans take radices 2-5."""
import pytest

import feram_b200 as fb
import helpers
import oracle_lib
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,prec", [("256 256 4", A.FG_PREC_MIXED), ("192 192 4", A.FG_PREC_MIXED),
                                    ("192 192 4", A.FG_PREC_FP64)])
def test_planes_that_do_not_fit_are_refused(fg, L, prec):
    p = helpers.params(L=L)
    with pytest.raises(fb.FeramError) as ei:
        fb.Context(p, prec)
    assert ei.value.code == A.FG_ERR_UNSUPPORTED and "shared memory" in str(ei.value)


def test_lengths_with_other_prime_factors_are_refused(fg):
    p = helpers.params(L="14 14 14")  # Lx/2 = 7
    with pytest.raises(fb.FeramError) as ei:
        fb.Context(p, A.FG_PREC_MIXED)
    assert ei.value.code == A.FG_ERR_UNSUPPORTED


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_largest_plane_matches_oracle(fg, prec):
    """160 x 160 x 4 (runtime-plan xy kernels: 80-point x and 160-point y
    transforms with a radix-5 stage): force and energies against the oracle
    at the precision's bar (mixed on an FP32-exact configuration)."""
    p = helpers.params(L="160 160 4", kelvin="250")
    u = helpers.seeded_u(p, 31, sigma=0.06)
    if prec == A.FG_PREC_MIXED:
        u = helpers.fp32_config(u)
    o = oracle_lib.Oracle(p)
    o.set_state(u)
    eo = o.force()
    with fb.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u)
        eg = ctx.mirror_force_mirror()
        fmax, frms = helpers.force_error(ctx.get_state()["dVddi"], o.get_state()["dVddi"], p)
    ee = helpers.energy_errors(eg, eo)
    ftol, etol = (1e-12, 1e-12) if prec == A.FG_PREC_FP64 else (1e-6, 1e-5)
    assert fmax <= ftol and frms <= ftol and max(ee.values()) <= etol, (fmax, frms, ee)
