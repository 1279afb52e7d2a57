"""Nose-Poincare Hamiltonian over 1e5 steps (16^3 BaTiO3, 200 K, dt 2 fs,
Q_Nose 0.1, GPa -5 as the reference's cooling example): the mixed-precision
path conserves H_NP as well as the FP64 path, whose per-step arithmetic is the
reference's (nose-poincare.F:10-78, energy_module.F:128-148; parity with the
oracle to 1e-11 per step in the other tests).  H_NP = s (H - H0) starts at 0,
settles into a bounded O(dt^2) excursion within the first few hundred steps
and must not drift after that."""
import numpy as np
import pytest

import helpers
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu

N_CHUNK, CHUNK = 200, 500  # 1e5 steps, H_NP sampled every 500


def _trace(fg, prec):
    p = helpers.params(L="16 16 16", kelvin="200", Q_Nose="0.1", GPa="-5.0")
    u = helpers.seeded_u(p, 7, sigma=0.02)
    with fg.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u)
        e = ctx.mirror_force_mirror()
        e.dipo_kinetic = ctx.kinetic_energy_dipo()
        ctx.nose_poincare_hamiltonian(e)
        ctx.set_thermostat(1.0, 0.0, e.H_Nose_Poincare)
        h, ke = [], []
        for _ in range(N_CHUNK):
            e = ctx.run_steps(CHUNK)
            h.append(e.H_Nose_Poincare)
            ke.append(e.dipo_kinetic / ctx.get_state()["s"] ** 2)  # real momenta p/s
    return np.array(h), np.array(ke), p


def test_hnp_drift_over_1e5_steps_mixed_no_worse_than_fp64(fg):
    h64, ke64, p = _trace(fg, A.FG_PREC_FP64)
    hmx, kemx, _ = _trace(fg, A.FG_PREC_MIXED)
    kT = 1.5 * p.N * p.temperature_eV  # target kinetic energy
    for h, ke in ((h64, ke64), (hmx, kemx)):
        assert np.all(np.isfinite(h))
        # thermostatted: the real kinetic energy of the last half sits at 3/2 N k T
        assert abs(ke[N_CHUNK // 2:].mean() - kT) < 0.05 * kT, (ke[N_CHUNK // 2:].mean(), kT)
        # bounded excursion, a small fraction of the kinetic energy
        assert np.abs(h).max() < 0.01 * kT, np.abs(h).max()
    drift = lambda h: h[-20:].mean() - h[:20].mean()
    assert abs(drift(hmx)) <= 2.0 * abs(drift(h64)) + 0.002 * kT, (drift(hmx), drift(h64))
    assert np.abs(hmx).max() <= 1.25 * np.abs(h64).max(), (np.abs(hmx).max(), np.abs(h64).max())
