"""Sweep points chained on the device (fg_chain_point) and the full-precision
.coord / .restart round trip (fg_write_coord, the .restart reader of
fg_feram_run), against the oracle replaying the reference's own chaining:
the previous point's final .coord, holding dipoP / s_Nose
(coord_module.F:476), read as .restart (initialize-dipoR.F:22-38), s = 1,
pi = 0 (:62-68) and H0 from that state (molecular-dynamics.F:52-55)."""
import numpy as np
import pytest

import helpers
import oracle_lib
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu


def _oracle_restart(p, u, q_over_s, n_steps):
    """A new oracle point from (u, p / s): initialize_dipoR's restart branch,
    then molecular_dynamics with H0 from that state."""
    o = oracle_lib.Oracle(p)
    o.set_state(u, q_over_s, 1.0, 0.0, 0.0)
    o.set_uniform_E(list(p.external_E_field))
    e = o.force()
    e.dipo_kinetic = o.kinetic_energy_dipo()
    o.md(1, n_steps, 1, e)
    return o, e


def test_chain_point_matches_oracle_restart(fg):
    """300 K for 12 steps, then the 280 K point from the device state, 12
    more steps: FP64 device path against the oracle at 1e-11."""
    p1 = helpers.params(L="8 8 8", kelvin="300")
    p2 = helpers.params(L="8 8 8", kelvin="280")
    u = helpers.seeded_u(p1, 4, sigma=0.06)
    q = helpers.seeded_p(p1, 4, sigma=0.02)
    o1 = oracle_lib.Oracle(p1)
    o1.set_state(u, q)
    e1 = o1.force()
    e1.dipo_kinetic = o1.kinetic_energy_dipo()
    o1.md(1, 12, 1, e1)
    s1 = o1.get_state()
    assert abs(s1["s"] - 1.0) > 1e-6  # the thermostat has moved: p / s matters
    o2, e2 = _oracle_restart(p2, s1["dipoR"], s1["dipoP"] / s1["s"], 12)
    s2 = o2.get_state()
    with fg.Context(p1, A.FG_PREC_FP64) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        e = ctx.mirror_force_mirror()
        e.dipo_kinetic = ctx.kinetic_energy_dipo()
        ctx.nose_poincare_hamiltonian(e)
        ctx.set_thermostat(1.0, 0.0, e.H_Nose_Poincare)
        ctx.run_steps(12)
        g1 = ctx.get_state()
        assert abs(g1["s"] - s1["s"]) <= 1e-12
        e0 = ctx.chain_point(280.0)
        assert ctx.p.kelvin == 280.0
        assert e0.H_Nose_Poincare == 0.0
        eg = ctx.run_steps(12)
        g2 = ctx.get_state()
    du = np.abs(A.physical(g2["dipoR"], p2) - A.physical(s2["dipoR"], p2)).max()
    dp = np.abs(A.physical(g2["dipoP"], p2) - A.physical(s2["dipoP"], p2)).max()
    assert du <= 1e-11 and dp <= 1e-11, (du, dp)
    assert abs(g2["s"] - s2["s"]) <= 1e-12 and abs(g2["pi"] - s2["pi"]) <= 1e-11
    assert abs(g2["H0"] - s2["H0"]) <= 1e-9 * abs(s2["H0"])
    for f in ("total", "unharmonic", "long_range", "dipo_kinetic", "H_Nose_Poincare"):
        a, b = getattr(eg, f), getattr(e2, f)
        assert abs(a - b) <= 1e-9 * max(abs(b), 1.0), (f, a, b)


@pytest.mark.parametrize("full", [True, False])
def test_write_coord_and_restart_reader(fg, tmp_path, full):
    """fg_write_coord of a stepped state, read back by fg_feram_run as
    <name>.restart; the run against the oracle started from the same file
    (parsed here as initialize-dipoR.F:27-34 reads it).  The full-precision
    file restarts the same state exactly; the reference's columns round u to
    1e-6 A and p to 7 digits."""
    p = helpers.params(L="8 8 8", kelvin="270")
    u = helpers.seeded_u(p, 6, sigma=0.06)
    q = helpers.seeded_p(p, 6, sigma=0.02)
    with fg.Context(p, A.FG_PREC_FP64) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        e = ctx.mirror_force_mirror()
        e.dipo_kinetic = ctx.kinetic_energy_dipo()
        ctx.nose_poincare_hamiltonian(e)
        ctx.set_thermostat(1.0, 0.0, e.H_Nose_Poincare)
        ctx.run_steps(9)
        st = ctx.get_state()
        ctx.write_coord(str(tmp_path / "run.restart"), full_precision=full)
    rows = np.loadtxt(tmp_path / "run.restart")
    assert rows.shape == (p.N, 18)
    got_u = rows[:, 3:6].reshape(p.Lz, p.Ly, p.Lx, 3)
    got_q = rows[:, 6:9].reshape(p.Lz, p.Ly, p.Lx, 3)
    ref_u = A.physical(st["dipoR"], p)
    ref_q = A.physical(st["dipoP"], p) / st["s"]
    if full:
        assert np.array_equal(got_u, ref_u) and np.array_equal(got_q, ref_q)
    else:
        assert np.abs(got_u - ref_u).max() <= 5.1e-7
        assert np.abs(got_q - ref_q).max() <= 1e-6 * np.abs(ref_q).max()
    # a run of the next point reads the file as its .restart
    n_th, n_av = 5, 6
    text = helpers.deck("zzznp.feram", L="8 8 8", kelvin="260", n_thermalize=str(n_th), n_average=str(n_av),
                        verbose="1", coord_directory="'never'")
    (tmp_path / "run.feram").write_text(text)
    avg, _ = fg.feram_run(str(tmp_path / "run.feram"), A.FG_PREC_FP64)
    p2 = fg.params_from_text(text, "run")
    u0, q0 = A.real_field(p2), A.real_field(p2)
    A.physical(u0, p2)[...] = got_u
    A.physical(q0, p2)[...] = got_q
    o = oracle_lib.Oracle(p2)
    o.set_state(u0, q0, 1.0, 0.0, 0.0)
    e = o.force()
    e.dipo_kinetic = o.kinetic_energy_dipo()
    ao = A.fg_average()
    o.md(1, n_th + n_av, 1, e, ao)
    assert avg.n_steps == ao.n_steps == n_av
    for f in ("total", "unharmonic", "long_range", "dipo_kinetic"):
        a, b = getattr(avg.energy, f), getattr(ao.energy, f)
        assert abs(a - b) <= 1e-9 * max(abs(b), 1.0), (f, a, b)
    for i in range(3):
        assert abs(avg.u[i] - ao.u[i]) <= 1e-9 * max(abs(ao.u[i]), 1.0)
