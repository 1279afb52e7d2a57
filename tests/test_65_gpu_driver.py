"""The host driver (fg_feram_run) for the methods and outputs beyond plain
Nose-Poincare: velocity scaling ('vs'), the hysteresis loop ('hl',
hysteresis_loop.F), the .hl lines of a field sweep, write_system's .coord
files (coord_module.F:434-486) and .dipoRavg (coord_module.F:578-608),
each checked against the oracle replaying the same sequence."""
import numpy as np
import pytest

import helpers
import oracle_lib
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu


def _run(fg, tmp_path, **tags):
    text = helpers.deck("zzznp.feram", **tags)
    (tmp_path / "run.feram").write_text(text)
    avg, _ = fg.feram_run(str(tmp_path / "run.feram"), A.FG_PREC_FP64)
    return avg, fg.params_from_text(text, "run")


def _rows(path):
    return np.array([[float(v) for v in line.split()] for line in path.read_text().splitlines() if line.strip()])


def test_feram_run_velocity_scaling_matches_oracle(fg, tmp_path):
    avg, p = _run(fg, tmp_path, L="8 8 8", method="'vs'", n_thermalize="6", n_average="8", verbose="1",
                  kelvin="260")
    o = oracle_lib.Oracle(p)
    e = o.initialize()
    ao = A.fg_average()
    o.md(1, p.n_thermalize + p.n_average, 0, e, ao)
    assert avg.n_steps == ao.n_steps == 8
    for f in ("total", "unharmonic", "long_range", "dipo_kinetic"):
        a, b = getattr(avg.energy, f), getattr(ao.energy, f)
        assert abs(a - b) <= 1e-9 * max(abs(b), 1.0), (f, a, b)
    for i in range(3):
        assert abs(avg.u[i] - ao.u[i]) <= 1e-9 * max(abs(ao.u[i]), 1.0)


def test_feram_run_hysteresis_loop_matches_oracle(fg, tmp_path):
    """hysteresis_loop.F:44-98: E ramps from +E to -E over n_average steps of
    velocity scaling; every n_hl_freq steps a .hl line (step, T, E, strain,
    <u>) and the .coord snapshot."""
    n_th, n_av, freq = 4, 8, 2
    _, p = _run(fg, tmp_path, L="8 8 8", method="'hl'", n_thermalize=str(n_th), n_average=str(n_av),
                n_hl_freq=str(freq), external_E_field="0.0 0.0 0.002", kelvin="150", verbose="1",
                coord_directory="''")
    lines = (tmp_path / "run.hl").read_text().splitlines()
    assert len(lines) == n_av // freq + 1
    o = oracle_lib.Oracle(p)
    e = o.initialize()
    expect = []
    for i_step in range(1, n_th + n_av + 1):
        if i_step >= n_th:
            E = [x - 2 * x * (i_step - n_th) / n_av for x in p.external_E_field]
            o.set_uniform_E(E)
        o.velocity_scaling(e)
        if i_step >= n_th and (i_step - n_th) % freq == 0:
            st = o.get_state()
            u = A.physical(st["dipoR"], p).reshape(-1, 3).mean(axis=0)
            expect.append((i_step, E, list(st["strain"]), u))
    for line, (i_step, E, strain, u) in zip(lines, expect):
        assert line[:10] == f"{i_step:010d}", line
        vals = [float(v) for v in line[10:].split()]
        assert vals[0] == pytest.approx(p.kelvin)
        assert np.allclose(vals[1:4], E, atol=1e-12)
        got = np.array(vals[4:13])
        ref = np.array(strain + list(u))
        assert np.allclose(got, ref, rtol=1e-4, atol=1e-9), (got, ref)  # E13.5: 5 significant digits
    # the last .hl line's snapshot
    rows = _rows(tmp_path / "run.coord")
    assert rows.shape == (p.N, 18)
    st = o.get_state()
    ref_u = A.physical(st["dipoR"], p)
    got_u = rows[:, 3:6].reshape(p.Lz, p.Ly, p.Lx, 3)
    assert np.abs(got_u - ref_u).max() <= 1e-6


def test_feram_run_coord_and_dipoRavg(fg, tmp_path):
    """write_system at n_coord_freq and divide_and_write_dipoRavg against the
    oracle's trajectory: u, p/s, dVddi and the relaxed acoustic field in the
    reference's column formats."""
    n_th, n_av = 3, 4
    _, p = _run(fg, tmp_path, L="8 8 8", n_thermalize=str(n_th), n_average=str(n_av), n_coord_freq="7",
                coord_directory="''", verbose="1", kelvin="280")
    o = oracle_lib.Oracle(p)
    e = o.initialize()
    uavg = np.zeros((p.Lz, p.Ly, p.Lx, 3))
    for i_step in range(1, n_th + n_av + 1):
        o.md(i_step, i_step, 1 if i_step == 1 else 0, e)
        st = o.get_state()
        if i_step == 7:
            snap = (A.physical(st["dipoR"], p).copy(), A.physical(st["dipoP"], p) / st["s"],
                    A.physical(st["dVddi"], p).copy(), A.physical(o.acouR_for_coord(), p).copy())
        if i_step > n_th:
            uavg += A.physical(st["dipoR"], p)
    rows = _rows(tmp_path / "run.0000000007.coord")
    assert rows.shape == (p.N, 18)
    assert np.array_equal(rows[:p.Lx, 0], np.arange(p.Lx))
    grid = rows[:, 3:].reshape(p.Lz, p.Ly, p.Lx, 15)
    assert np.abs(grid[..., 0:3] - snap[0]).max() <= 1e-6
    for k, ref in ((1, snap[1]), (2, snap[2]), (3, snap[3])):
        got = grid[..., 3 * k:3 * k + 3]
        # E14.6 keeps 6 significant digits
        assert np.allclose(got, ref, rtol=1e-5, atol=1e-12 + 1e-6 * np.abs(ref).max()), k
    assert np.all(grid[..., 12:15] == 0.0)
    ravg = _rows(tmp_path / "run.dipoRavg")
    assert ravg.shape == (p.N, 6)
    assert np.abs(ravg[:, 3:].reshape(p.Lz, p.Ly, p.Lx, 3) - uavg / n_av).max() <= 1e-6


@pytest.mark.parametrize("zstar", ["9.956 9.956 9.956", "9.956 7.3 7.3"])
def test_feram_run_reads_relaxor_defects_localfield(fg, tmp_path, zstar):
    """initialize_dipoR's read_relaxor and read_defects_u and
    initialize_E_field's .localfield through the host driver, against the
    oracle given the same per-site arrays; species with equal and with
    different Z*."""
    text = helpers.deck("zzznp.feram", L="8 8 8", n_thermalize="4", n_average="6", verbose="1", kelvin="240",
                        P_kappa2="5.502 4.61 4.61", P_alpha="110.4 98.2 98.2", mass_amu="39.0 47.5 47.5",
                        Z_star=zstar)
    (tmp_path / "run.feram").write_text(text)
    p = fg.params_from_text(text, "run")
    rng = np.random.default_rng(8)
    rel = [(x, y, z, int(rng.integers(1, 3))) for z in range(8) for y in range(8) for x in range(8)]
    (tmp_path / "run.relaxor").write_text("# ix iy iz species\n" + "".join(f"{x} {y} {z} {r}\n" for x, y, z, r in rel))
    defects = [(1, 1, 1, 0.05, 0.0, -0.03), (6, 2, 5, 0.0, 0.07, 0.0)]
    (tmp_path / "run.defects").write_text("".join(f"{x} {y} {z} {a} {b} {c}\n" for x, y, z, a, b, c in defects))
    loc = [(x, y, 3, 0.0, 0.0, 0.004) for y in range(8) for x in range(8)]
    (tmp_path / "run.localfield").write_text("".join(f"{x} {y} {z} {a} {b} {c}\n" for x, y, z, a, b, c in loc))
    avg, _ = fg.feram_run(str(tmp_path / "run.feram"), A.FG_PREC_FP64)
    # the oracle with the same arrays
    shape = (p.Lz, p.Ly + p.padding_y, 2 * (p.Lx // 2 + 1))
    relaxor = np.ones(shape, dtype=np.int32)
    zs = np.full(shape, p.Z_star[0])
    minv = np.zeros(shape)
    sum_p = np.zeros(shape, dtype=np.int32)
    sum_p[:, :p.Ly, :p.Lx] = 1
    for x, y, z, r in rel:
        relaxor[z, y, x] = r
        zs[z, y, x] = p.Z_star[r - 1]
        minv[z, y, x] = 1.0 / p.mass_dipo[r - 1]
    eloc = A.real_field(p)
    for x, y, z, a, b, c in loc:
        A.physical(eloc, p)[z, y, x] = (a, b, c)
    o = oracle_lib.Oracle(p)
    o.initialize()
    st = o.get_state()
    u = st["dipoR"].copy()
    for x, y, z, a, b, c in defects:
        A.physical(u, p)[z, y, x] = (a, b, c)
        minv[z, y, x] = 0.0
        sum_p[z, y, x] = 0
    o.set_sites(Z_starR=zs, relaxor=relaxor, mass_dipo_inv=minv, sum_p=sum_p, E_field_local=eloc)
    o.set_state(u, st["dipoP"], 1.0, 0.0, 0.0)
    e = o.force()
    e.dipo_kinetic = o.kinetic_energy_dipo()
    ao = A.fg_average()
    o.md(1, p.n_thermalize + p.n_average, 1, e, ao)
    assert avg.n_steps == ao.n_steps == 6
    for f in ("total", "unharmonic", "dipole_E_field", "dipo_kinetic", "long_range"):
        a, b = getattr(avg.energy, f), getattr(ao.energy, f)
        assert abs(a - b) <= 1e-9 * max(abs(b), 1.0), (f, a, b)
    assert avg.energy.dipole_E_field != 0.0
    for i in range(3):
        assert abs(avg.u[i] - ao.u[i]) <= 1e-9 * max(abs(ao.u[i]), 1.0)
