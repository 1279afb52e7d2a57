"""Acoustic-displacement MD (acoustic_mass_amu > 0) on the device against the
oracle: acouFFT, dVdac, kinetic_energy_acou, the acoustic branches of
leapfrog (leapfrog.F:9-157) and velocity_scaling (velocity_scaling.F:86-98),
and the delta_e heat pump (leapfrog.F:44-87)."""
import numpy as np
import pytest

import helpers
import oracle_lib
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu

TOL = {A.FG_PREC_FP64: 1e-10, A.FG_PREC_MIXED: 2e-5}


def _rel(a, b, p):
    a, b = A.physical(a, p), A.physical(b, p)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _start(p, seed):
    u = helpers.seeded_u(p, seed, sigma=0.06, avg=0.05)
    q = helpers.seeded_p(p, seed, sigma=0.01)
    ar = helpers.seeded_u(p, seed + 77, sigma=0.003)
    ap = helpers.seeded_u(p, seed + 78, sigma=0.004)
    return u, q, ar, ap


def _compare(ctx, o, eg, eo, p, prec, tag):
    sg, so = ctx.get_state(), o.get_state()
    ag, ao = ctx.get_acou(), o.get_acou()
    err = {k: _rel(sg[k], so[k], p) for k in ("dipoR", "dipoP", "dVddi")}
    err.update({k: _rel(ag[k], ao[k], p) for k in ("acouR", "acouP", "dVdacR")})
    ee = helpers.energy_errors(eg, eo, A.POTENTIAL_FIELDS + ["dipo_kinetic", "acou_kinetic"])
    worst = max(list(err.values()) + list(ee.values()))
    assert worst <= TOL[prec], (tag, err, ee)


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
@pytest.mark.parametrize("L", ["16 16 16", "12 10 8"])
def test_leapfrog_acoustic_matches_oracle(fg, prec, L):
    p = helpers.params("zzzlf.feram", L=L, kelvin="200")
    assert p.mass_acou[0] > 0.0
    u, q, ar, ap = _start(p, 11)
    o = oracle_lib.Oracle(p)
    o.set_state(u, q)
    o.set_acou(ar, ap)
    eo = A.fg_energy()
    with fg.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        ctx.set_acou(ar, ap)
        eg = A.fg_energy()
        for step in range(0, 8):  # i_step 0 is the half-kick start
            o.leapfrog(eo, step)
            ctx.leapfrog(eg, step)
        _compare(ctx, o, eg, eo, p, prec, "lf")
        assert eg.acou_kinetic > 0.0


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_velocity_scaling_acoustic_matches_oracle(fg, prec):
    p = helpers.params("zzzlf.feram", L="16 16 16", method="'vs'", kelvin="220")
    u, q, ar, ap = _start(p, 12)
    o = oracle_lib.Oracle(p)
    o.set_state(u, q)
    o.set_acou(ar, ap)
    eo = o.force()
    with fg.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        ctx.set_acou(ar, ap)
        eg = ctx.mirror_force_mirror()
        for _ in range(5):
            o.velocity_scaling(eo)
            ctx.velocity_scaling(eg)
        _compare(ctx, o, eg, eo, p, prec, "vs")


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_leapfrog_heat_pump_matches_oracle(fg, prec):
    """delta_e and delta_e_acou scale the momenta of layers Lz/4 and 3 Lz/4."""
    p = helpers.params("zzzlf.feram", L="8 8 16", kelvin="250", delta_e="0.0002", delta_e_acou="0.0001")
    u, q, ar, ap = _start(p, 13)
    o = oracle_lib.Oracle(p)
    o.set_state(u, q)
    o.set_acou(ar, ap)
    eo = A.fg_energy()
    with fg.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        ctx.set_acou(ar, ap)
        eg = A.fg_energy()
        for step in range(0, 6):
            o.leapfrog(eo, step)
            ctx.leapfrog(eg, step)
        _compare(ctx, o, eg, eo, p, prec, "pump")


def test_acoustic_with_modulation_matches_oracle(fg):
    p = helpers.params("zzzlf.feram", L="16 16 16", modulation_constant="6.3")
    u, q, ar, ap = _start(p, 14)
    rng = np.random.default_rng(14)
    mod = np.zeros((p.Lz, p.Ly + p.padding_y, 2 * (p.Lx // 2 + 1)))
    mod[:, :p.Ly, :p.Lx] = rng.standard_normal((p.Lz, p.Ly, p.Lx)) * 0.01
    o = oracle_lib.Oracle(p)
    o.set_modulation_R(mod)
    o.set_state(u, q)
    o.set_acou(ar, ap)
    eo = o.force()
    with fg.Context(p, A.FG_PREC_FP64) as ctx:
        ctx.build_tables()
        ctx.set_modulation_R(mod)
        ctx.set_state(u, q)
        ctx.set_acou(ar, ap)
        eg = ctx.mirror_force_mirror()
        _compare(ctx, o, eg, eo, p, A.FG_PREC_FP64, "modulation")
