"""Ensemble averages against the reference's own published run: the first
point (350 K, paraelectric) of the 16^3 cooling sweep of
src/03example-BaTiO3-bulk-phase-transition/16x16x16-40000-10000
(cooling.sh: GPa = -5, Q_Nose = 0.1, 40000 + 10000 Nose-Poincare steps from
the uni64-seeded start), committed as tests/golden/cooling16.json.  The
trajectories are chaotic, so only averages compare; the tolerances are a few
times the deviations seen between independent runs and the reference's own
scatter between neighbouring temperatures."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import helpers
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "cooling16.json")))

# column -> (absolute tolerance, relative tolerance); .avg columns of
# average_module.F:243-260 up to dipo_kinetic_true
TOL = {
    4: (1.5e-4, 0), 5: (1.5e-4, 0), 6: (1.5e-4, 0),        # strain 1..3
    7: (2e-5, 0), 8: (2e-5, 0), 9: (2e-5, 0),              # strain 4..6
    10: (1e-2, 0), 11: (1e-2, 0), 12: (1e-2, 0),           # <u>
    19: (0, 2e-2),                                         # dipo_kinetic
    22: (3e-4, 0), 23: (3e-4, 0), 24: (5e-4, 0),           # unharmonic, homo_strain, homo_coupling
    25: (1e-4, 0), 26: (2e-4, 0), 27: (3e-4, 0),           # inho_strain, inho_coupling, total
    30: (0, 1e-2),                                         # dipo_kinetic_true (3/2 k T)
}


@pytest.mark.parametrize("prec", [A.FG_PREC_MIXED, A.FG_PREC_FP64])
def test_cooling_350K_averages_match_reference(fg, tmp_path, prec):
    row = GOLD["rows"][0]
    assert row[0] == 350.0
    text = helpers.deck("zzznp.feram", L="16 16 16", kelvin="350", GPa="-5.0", Q_Nose="0.1",
                        n_thermalize=str(GOLD["n_thermalize"]), n_average=str(GOLD["n_average"]),
                        init_dipo_avg="0.0 0.0 0.0", init_dipo_dev="0.03 0.03 0.03", verbose="1",
                        coord_directory="'never'")
    (tmp_path / "c350.feram").write_text(text)
    fg.feram_run(str(tmp_path / "c350.feram"), prec)
    got = [float(v) for v in (tmp_path / "c350.avg").read_text().split()]
    assert len(got) == 43
    for col, (atol, rtol) in TOL.items():
        assert abs(got[col] - row[col]) <= atol + rtol * abs(row[col]), (col, got[col], row[col])
    # the 2012 .avg of the golden reported the whole dipole-dipole energy in
    # its long_range column; today's reference splits it into long_range and
    # short_range (column 32)
    assert abs(got[20] + got[32] - row[20]) <= 1e-3, (got[20], got[32], row[20])
    for col in (13, 14, 15):  # (sum u)^2 / N: fluctuation size, paraelectric
        assert 0.0 < got[col] < 1.0


def _jackknife(blocks, fn):
    """Value of fn over all blocks and its jackknife standard error."""
    B = len(blocks)
    full = fn(np.concatenate(blocks))
    loo = np.array([fn(np.concatenate(blocks[:b] + blocks[b + 1:])) for b in range(B)])
    return full, np.sqrt((B - 1) / B * np.sum((loo - loo.mean(axis=0)) ** 2, axis=0))


def test_cooling_chain_to_200K_ordered_phase_matches_reference(fg):
    """The reference's 16^3 cooling sweep (cooling.sh: 350 K down to 200 K
    in 5 K steps, 40000 + 10000 Nose-Poincare steps per point, each point
    started from the previous one's final state) with the points chained on
    the device (fg_chain_point), mixed precision.  At 200 K (cooling.avg,
    rhombohedral phase: <u> ~ 0.087 A on every axis) the averages are
    compared with block-averaged (jackknife, 10 and 5 blocks) error bars of this
    run: |<u_a>| and the diagonal strains (sorted: the polar axis of the
    ordered state is chosen by the trajectory), the susceptibility
    chi_a ~ ((sum u_a)^2/N - N <u_a>^2) / T of strain-susceptibility.gp:36-59
    averaged over the axes, and the energies.  Tolerance: 4 sigma of the
    difference of two independent runs (sqrt 2 times this run's sigma, the
    larger of its 10- and 5-block jackknife errors) plus the rounding of the
    .avg's printed digits."""
    gold = {r[0]: r for r in GOLD["rows"]}
    n_th, n_av = GOLD["n_thermalize"], GOLD["n_average"]
    p = helpers.params("zzznp.feram", L="16 16 16", kelvin="350", GPa="-5.0", Q_Nose="0.1",
                       init_dipo_avg="0.0 0.0 0.0", init_dipo_dev="0.03 0.03 0.03")
    N = p.N
    with fg.Context(p, A.FG_PREC_MIXED) as ctx:
        ctx.build_tables()
        u0, q0 = A.real_field(p), A.real_field(p)
        assert A.lib().fg_init_dipoR_host(C.byref(p), A.dptr(u0), A.dptr(q0)) == 0
        ctx.set_state(u0, q0)
        e = ctx.mirror_force_mirror()
        e.dipo_kinetic = ctx.kinetic_energy_dipo()
        ctx.nose_poincare_hamiltonian(e)
        ctx.set_thermostat(1.0, 0.0, e.H_Nose_Poincare)
        temps = [350.0 - 5.0 * i for i in range(31)]
        for i, T in enumerate(temps):
            if i > 0:
                ctx.chain_point(T)
            if T > 200.0:
                ctx.run_steps(n_th + n_av)
        # the 200 K point: thermalise, then per-step sums for block averages
        e = ctx.run_steps(n_th)
        avg = A.fg_average()
        su, en, st = [], [], []
        prev_u, prev_s, prev_k = np.zeros(3), np.zeros(6), 0.0
        for _ in range(n_av):
            ctx.run_steps(1, e)
            ctx.average_accumulate(e, avg)
            cur_u, cur_s = np.array(avg.u[:]), np.array(avg.strain[:])
            su.append(cur_u - prev_u)  # sum over sites of u this step
            st.append(cur_s - prev_s)  # this step's homogeneous strain
            kt = avg.dipo_kinetic_true - prev_k  # KE / s^2 this step
            prev_u, prev_s, prev_k = cur_u, cur_s, avg.dipo_kinetic_true
            en.append([kt, e.unharmonic, e.homo_strain, e.homo_coupling, e.inho_strain, e.inho_coupling, e.total])
    su, en, st = np.array(su), np.array(en), np.array(st)
    row = gold[200.0]

    def blocked(a, fn):
        # the larger of the jackknife errors over 10 and over 5 blocks: the
        # homogeneous strain and its energy stay correlated over more than
        # 1000 steps, which the longer blocks take in (Flyvbjerg-Petersen
        # blocking: the error grows with the block until blocks decorrelate)
        out = []
        for nb in (10, 5):
            blk = [a[i * (n_av // nb):(i + 1) * (n_av // nb)] for i in range(nb)]
            out.append(_jackknife(blk, fn))
        return out[0][0], np.maximum(out[0][1], out[1][1])
    u_mean, u_err = blocked(su, lambda s: np.sort(np.abs(s.mean(axis=0))) / N)
    chi, chi_err = blocked(su, lambda s: np.mean((s ** 2).mean(axis=0) / N - (s.mean(axis=0)) ** 2 / N))
    e_mean, e_err = blocked(en, lambda a: a.mean(axis=0))
    s_mean, s_err = blocked(st, lambda a: np.sort(a.mean(axis=0)[:3]))
    ref_u = np.sort(np.abs(np.array(row[10:13])))
    ref_chi = np.mean(np.array(row[13:16]) - N * np.array(row[10:13]) ** 2)
    ref_s = np.sort(np.array(row[4:7]))
    k = 4.0 * np.sqrt(2.0)
    bad = []
    if not np.all(np.abs(u_mean - ref_u) <= k * u_err + 1e-5):
        bad.append(("|<u>|", u_mean, u_err, ref_u))
    if not np.all(np.abs(s_mean - ref_s) <= k * s_err + 1e-6):
        bad.append(("strain", s_mean, s_err, ref_s))
    if not abs(chi - ref_chi) <= k * chi_err + 3e-3:
        bad.append(("chi", chi, chi_err, ref_chi))
    # the .avg energies are per site (average_module.F:198-199); column 30 is
    # the kinetic energy KE / s^2 (dipo_kinetic_true), the physical one; the
    # Nose-scaled column 19 depends on the thermostat's s and is not compared
    for j, col in enumerate((30, 22, 23, 24, 25, 26, 27)):
        em, ee = e_mean[j] / N, e_err[j] / N
        if not abs(em - row[col]) <= k * ee + 1e-5 * abs(row[col]) + 1e-7:
            bad.append((col, em, ee, row[col]))
    assert not bad, bad
