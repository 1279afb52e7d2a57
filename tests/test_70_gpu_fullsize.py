"""Full-size checks: the compile-time FFT instances (32^3 .. 128^3) against
numpy and the oracle, and size-independent properties at 128^3.

Force parity at full size: FP64 worst site and RMS of |dF| <= 1e-12 of
RMS |F| and every energy term <= 1e-12; mixed worst site and RMS <= 1e-6
(on the FP32-rounded configuration both paths hold), energies <= 1e-5.
Measured errors go to FERAM_PARITY_LOG when it is set."""
import json
import os

import numpy as np
import pytest

import helpers
import oracle_lib
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu

TOL = {A.FG_PREC_FP64: 2e-13, A.FG_PREC_MIXED: 3e-6}


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
@pytest.mark.parametrize("L", [32, 64, 128])
def test_fft_roundtrip_fullsize(fg, L, prec):
    p = helpers.params(L=f"{L} {L} {L}")
    with fg.Context(p, prec) as ctx:
        rng = np.random.default_rng(L)
        f = A.real_field(p)
        A.physical(f, p)[...] = rng.standard_normal((L, L, L, 3))
        X = ctx.fft_r2c3(f)
        ref = np.fft.rfftn(A.physical(f, p), axes=(0, 1, 2))
        err = np.abs(X[:, :L] - ref).max() / np.abs(ref).max()
        assert err <= TOL[prec], err
        back = ctx.fft_c2r3(X)
        err2 = np.abs(A.physical(back, p) / p.N - A.physical(f, p)).max() / np.abs(A.physical(f, p)).max()
        assert err2 <= TOL[prec] * 5, err2


LOG = os.environ.get("FERAM_PARITY_LOG")


def _record(name, data):
    if not LOG:
        return
    os.makedirs(os.path.dirname(os.path.abspath(LOG)), exist_ok=True)
    with open(LOG, "a") as f:
        f.write(json.dumps({"test": name, **data}) + "\n")


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
@pytest.mark.parametrize("Ez", [0.0, 0.001])
@pytest.mark.parametrize("L", [32, 64, 128])
def test_force_matches_oracle_fullsize(fg, L, Ez, prec):
    """The 128^3 workload at E_z = 0 and 100 kV/cm (0.001 V/A)."""
    p = helpers.params(L=f"{L} {L} {L}", external_E_field=f"0.0 0.0 {Ez}")
    u = helpers.seeded_u(p, 100 + L, sigma=0.1)
    if prec == A.FG_PREC_MIXED:
        u = helpers.fp32_config(u)
    o = oracle_lib.Oracle(p)
    o.set_state(u)
    o.set_uniform_E([0.0, 0.0, Ez])
    eo = o.force()
    with fg.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u)
        ctx.set_uniform_E([0.0, 0.0, Ez])
        eg = ctx.mirror_force_mirror()
        fgd = ctx.get_state()["dVddi"]
    fmax, frms = helpers.force_error(fgd, o.get_state()["dVddi"], p)
    ee = helpers.energy_errors(eg, eo)
    _record(f"force_fullsize[{L},{Ez},{prec}]", dict(fmax=fmax, frms=frms, emax=max(ee.values()),
                                                      energies={k: float(v) for k, v in ee.items()}))
    if prec == A.FG_PREC_FP64:
        assert fmax <= 1e-12 and frms <= 1e-12 and max(ee.values()) <= 1e-12, (fmax, ee)
    else:
        assert frms <= 1e-6 and fmax <= 1e-6 and max(ee.values()) <= 1e-5, (fmax, frms, ee)


def test_nose_poincare_128_matches_oracle(fg):
    p = helpers.params(L="128 128 128", Q_Nose="8.0", kelvin="300")
    u = helpers.seeded_u(p, 7, sigma=0.05)
    q = helpers.seeded_p(p, 7, sigma=0.01)
    o = oracle_lib.Oracle(p)
    o.set_state(u, q)
    eo = o.force()
    eo.dipo_kinetic = o.kinetic_energy_dipo()
    with fg.Context(p, A.FG_PREC_FP64) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        eg = ctx.mirror_force_mirror()
        eg.dipo_kinetic = ctx.kinetic_energy_dipo()
        for _ in range(3):
            o.nose_poincare(eo)
            ctx.nose_poincare(eg)
        sg = ctx.get_state()
    so = o.get_state()
    du = np.abs(A.physical(sg["dipoR"], p) - A.physical(so["dipoR"], p)).max() / np.abs(A.physical(so["dipoR"], p)).max()
    ee = helpers.energy_errors(eg, eo, A.POTENTIAL_FIELDS + ["dipo_kinetic", "H_Nose_Poincare"])
    assert du <= 1e-11 and abs(sg["s"] - so["s"]) <= 1e-12, (du, sg["s"], so["s"])
    assert max(v for k, v in ee.items() if k != "H_Nose_Poincare") <= 1e-10, ee


def test_nose_poincare_128_second_order(fg):
    """H_NP is conserved up to a bounded O(dt^2) excursion (nose-poincare.F is
    the symplectic generalised leapfrog): halving dt quarters the excursion."""
    peaks = []
    for dt, n in ((0.002, 60), (0.001, 120)):
        p = helpers.params(L="128 128 128", Q_Nose="8.0", kelvin="300", dt=str(dt))
        u = helpers.seeded_u(p, 5, sigma=0.05)
        with fg.Context(p, A.FG_PREC_FP64) as ctx:
            ctx.build_tables()
            ctx.set_state(u)
            e = ctx.mirror_force_mirror()
            e.dipo_kinetic = ctx.kinetic_energy_dipo()
            ctx.nose_poincare_hamiltonian(e)
            ctx.set_thermostat(1.0, 0.0, e.H_Nose_Poincare)
            h = 0.0
            for _ in range(n):
                ctx.nose_poincare(e)
                h = max(h, abs(e.H_Nose_Poincare))
        peaks.append(h)
    assert 3.5 < peaks[0] / peaks[1] < 4.5, peaks


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_harmonic_force_is_linear_128(fg, prec):
    """With the anharmonic and strain-coupling constants set to zero the force
    is linear in u: F(u1 + 2 u2) = F(u1) + 2 F(u2)."""
    p = helpers.params(L="128 128 128", P_alpha="0.0", P_gamma="0.0", B1xx="0.0", B1yy="0.0", B4yz="0.0")
    u1 = helpers.seeded_u(p, 21, sigma=0.05)
    u2 = helpers.seeded_u(p, 22, sigma=0.05)
    with fg.Context(p, prec) as ctx:
        ctx.build_tables()
        F = []
        for u in (u1, u2, u1 + 2 * u2):
            ctx.set_state(u)
            ctx.mirror_force_mirror()
            F.append(A.physical(ctx.get_state()["dVddi"], p).copy())
    lhs, rhs = F[2], F[0] + 2 * F[1]
    err = np.abs(lhs - rhs).max() / np.abs(lhs).max()
    assert err <= (1e-12 if prec == A.FG_PREC_FP64 else 3e-6), err
