"""Force, energies and MD steps of the device path against the FP64 oracle.

FP64 device path: forces and every energy term within 1e-12 relative (RMS-
normalised forces, term-wise energies).  Mixed path (FP32 fields/FFT, FP64
site force sums, thermostat and strain): worst site and RMS of |dF| each
<= 1e-6 of RMS |F|, energies <= 1e-5 of the energy scale, measured on
configurations the mixed path can hold (u rounded to FP32, given to both).
"""
import json
import os

import numpy as np
import pytest

import helpers
import oracle_lib
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu

FTOL = {A.FG_PREC_FP64: 1e-12, A.FG_PREC_MIXED: 1e-6}
ETOL = {A.FG_PREC_FP64: 1e-12, A.FG_PREC_MIXED: 1e-5}
# measured errors appended as JSON lines to this file when it is set
LOG = os.environ.get("FERAM_PARITY_LOG")

CASES = {
    "zvr16": dict(base="zzznp.feram", L="16 16 16"),
    "new16": dict(base="zzz16.feram", L="16 16 16"),
    "odd": dict(base="zzznp.feram", L="20 12 18"),
    "efield": dict(base="zzznp.feram", L="16 16 16", external_E_field="0.0005 -0.0002 0.001"),
    "epit": dict(base="zzznp.feram", L="12 12 8", bulk_or_film="'epit'", epi_strain="0.01"),
    "film_gap": dict(base="zzznp.feram", L="12 10 9", bulk_or_film="'film'", gap_id="1",
                     gap_dipole_u="0.0 0.0 0.05"),
}


def _record(name, data):
    if not LOG:
        return
    os.makedirs(os.path.dirname(os.path.abspath(LOG)), exist_ok=True)
    with open(LOG, "a") as f:
        f.write(json.dumps({"test": name, **data}) + "\n")


def _setup(fg, case, prec, seed, tables="build"):
    c = dict(CASES[case])
    base = c.pop("base")
    p = helpers.params(base, **c)
    o = oracle_lib.Oracle(p)
    ctx = fg.Context(p, prec)
    if tables == "build":
        ctx.build_tables()
    else:
        ctx.upload_tables(*o.tables())
    u = helpers.seeded_u(p, seed, sigma=0.1)
    if p.gap_id > 0:  # dead layers hold gap_dipole_u (read_defects_u.F:56-69)
        for z in ([0] if p.gap_id == 1 else [0, p.Lz // 2]):
            u[z, :p.Ly, :p.Lx, :] = np.array(list(p.gap_dipole_u))
    if prec == A.FG_PREC_MIXED:
        u = helpers.fp32_config(u)
    return p, o, ctx, u


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("tables", ["build", "upload"])
def test_force_and_energies_match_oracle(fg, case, prec, tables):
    p, o, ctx, u = _setup(fg, case, prec, seed=1 + list(CASES).index(case), tables=tables)
    E = np.array(list(p.external_E_field))
    o.set_state(u)
    ctx.set_state(u)
    if not p.E_field_always_zero:
        o.set_uniform_E(E)
        ctx.set_uniform_E(E)
    eo = o.force()
    eg = ctx.mirror_force_mirror()
    so, sg = o.get_state(), ctx.get_state()
    fmax, frms = helpers.force_error(sg["dVddi"], so["dVddi"], p)
    ee = helpers.energy_errors(eg, eo)
    serr = float(np.abs(sg["strain"] - so["strain"]).max() / max(np.abs(so["strain"]).max(), 1e-30))
    _record(f"force[{case},{prec},{tables}]", dict(fmax=fmax, frms=frms, emax=max(ee.values()), strain=serr,
                                                   energies={k: float(v) for k, v in ee.items()}))
    # the film mirror rewrites the upper half of u: the device must agree
    assert np.abs(A.physical(sg["dipoR"], p) - A.physical(so["dipoR"], p)).max() <= FTOL[prec]
    assert fmax <= FTOL[prec], (fmax, frms)
    assert frms <= FTOL[prec]
    assert max(ee.values()) <= ETOL[prec], ee
    assert serr <= ETOL[prec]
    ctx.close()


def test_modulation_acouK_and_energies(fg):
    k = helpers.golden("modulation_kat.json")
    p = fg.params_from_text(k["feram"], "zzzmodulation")
    mod = np.zeros((p.Lz, p.Ly + p.padding_y, 2 * (p.Lx // 2 + 1)))
    for ix, iy, iz, v in k["modulation"]:
        mod[int(iz), int(iy), int(ix)] = v
    o = oracle_lib.Oracle(p)
    o.set_modulation_R(mod)
    u = helpers.seeded_u(p, 9, sigma=0.05)
    o.set_state(u)
    eo = o.force()
    with fg.Context(p, A.FG_PREC_FP64) as ctx:
        ctx.build_tables()
        ctx.set_modulation_R(mod)
        ctx.set_state(u)
        eg = ctx.mirror_force_mirror()
        ag = ctx.get_acouK()
        fg_state = ctx.get_state()
    ao = o.acouK()
    aerr = np.abs(ag[:, :p.Ly] - ao[:, :p.Ly]).max() / np.abs(ao).max()
    fmax, _ = helpers.force_error(fg_state["dVddi"], o.get_state()["dVddi"], p)
    ee = helpers.energy_errors(eg, eo)
    _record("modulation", dict(acouK=float(aerr), fmax=fmax, emax=max(ee.values())))
    assert aerr <= 1e-11 and fmax <= 1e-11 and max(ee.values()) <= 1e-11, (aerr, fmax, ee)


def test_modulation_check_kat_on_device(fg, tmp_path):
    """modulation_check.sh through the host driver and the device path."""
    k = helpers.golden("modulation_kat.json")
    (tmp_path / "zzzmodulation.feram").write_text(k["feram"])
    (tmp_path / "zzzmodulation.modulation").write_text(
        "\n".join("%d %d %d %.1f" % (a, b, c, v) for a, b, c, v in k["modulation"]) + "\n")
    fg.feram_run(str(tmp_path / "zzzmodulation.feram"), A.FG_PREC_FP64)
    log = (tmp_path / "zzzmodulation.log").read_text().splitlines()
    strain = [l for l in log if l.startswith("inho_strain") and l.split()[1] == k["inho_strain_per_cell"]]
    modl = [l for l in log if l.startswith("inho_modulation") and l.split()[1] == k["inho_modulation_per_cell"]]
    assert len(strain) == k["n_log_lines"] and len(modl) == k["n_log_lines"], log[:40]


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_nose_poincare_steps_match_oracle(fg, prec):
    p = helpers.params(L="16 16 16", kelvin="250")
    o = oracle_lib.Oracle(p)
    u = helpers.seeded_u(p, 21, sigma=0.08)
    q = helpers.seeded_p(p, 21, sigma=0.01)  # thermal: sqrt(m kT) ~ 0.01
    o.set_state(u, q)
    eo = o.force()
    eo.dipo_kinetic = o.kinetic_energy_dipo()
    with fg.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        eg = ctx.mirror_force_mirror()
        eg.dipo_kinetic = ctx.kinetic_energy_dipo()
        # H0 from the initial state (molecular-dynamics.F:209-212)
        o.set_state(None, None, 1.0, 0.0, 0.0)
        h = o.L.oracle_nose_poincare_hamiltonian(o.h, __import__("ctypes").byref(eo))
        o.set_state(None, None, 1.0, 0.0, h)
        ctx.set_thermostat(1.0, 0.0, h)
        worst = {}
        for step in range(1, 21):
            o.nose_poincare(eo)
            ctx.nose_poincare(eg)
            if step % 5 == 0:
                so, sg = o.get_state(), ctx.get_state()
                du = np.abs(A.physical(sg["dipoR"], p) - A.physical(so["dipoR"], p)).max()
                dp = np.abs(A.physical(sg["dipoP"], p) - A.physical(so["dipoP"], p)).max()
                ru = du / np.abs(A.physical(so["dipoR"], p)).max()
                rp = dp / np.abs(A.physical(so["dipoP"], p)).max()
                ds = abs(sg["s"] - so["s"])
                ee = helpers.energy_errors(eg, eo, A.POTENTIAL_FIELDS + ["dipo_kinetic"])
                worst = dict(step=step, u=float(ru), p=float(rp), s=float(ds), e=float(max(ee.values())),
                             H=float(abs(eg.H_Nose_Poincare - eo.H_Nose_Poincare)))
    _record(f"np20[{prec}]", worst)
    tol = 1e-9 if prec == A.FG_PREC_FP64 else 2e-5
    assert worst["u"] <= tol and worst["p"] <= tol and worst["s"] <= tol and worst["e"] <= tol, worst


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_leapfrog_steps_match_oracle(fg, prec):
    p = helpers.params(L="12 10 8", method="'lf'")
    o = oracle_lib.Oracle(p)
    u = helpers.seeded_u(p, 31, sigma=0.08)
    o.set_state(u)
    eo = o.force()
    with fg.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u)
        eg = ctx.mirror_force_mirror()
        for step in range(1, 11):
            o.leapfrog(eo, step)
            ctx.leapfrog(eg, step)
        so, sg = o.get_state(), ctx.get_state()
    ru = np.abs(A.physical(sg["dipoR"], p) - A.physical(so["dipoR"], p)).max() / np.abs(A.physical(so["dipoR"], p)).max()
    ee = helpers.energy_errors(eg, eo, A.POTENTIAL_FIELDS + ["dipo_kinetic"])
    _record(f"lf10[{prec}]", dict(u=float(ru), e=float(max(ee.values()))))
    tol = 1e-10 if prec == A.FG_PREC_FP64 else 1e-5
    assert ru <= tol and max(ee.values()) <= tol, (ru, ee)


WAVE = dict(external_E_field="0.0 0.0 0.002", E_wave_type="'triangular_cos'", n_E_wave_period="8")


@pytest.mark.parametrize("extra", [{}, WAVE], ids=["static", "triangular_cos"])
def test_feram_run_matches_oracle_md(fg, tmp_path, extra):
    """The whole host driver (initialize_dipoR with uni64, H0, NP loop with
    the per-step field of wave_module.F, add_to_Average) against the
    oracle's molecular_dynamics."""
    text = helpers.deck("zzznp.feram", L="8 8 8", n_thermalize="10", n_average="10", verbose="1",
                        n_coord_freq="100000", kelvin="280", **extra)
    (tmp_path / "run.feram").write_text(text)
    avg, tsim = fg.feram_run(str(tmp_path / "run.feram"), A.FG_PREC_FP64)
    p = fg.params_from_text(text, "run")
    o = oracle_lib.Oracle(p)
    e = o.initialize()
    ao = A.fg_average()
    o.md(1, p.n_thermalize + p.n_average, 1, e, ao)
    assert avg.n_steps == ao.n_steps == 10
    for f in ("total", "unharmonic", "long_range", "dipo_kinetic", "H_Nose_Poincare"):
        a, b = getattr(avg.energy, f), getattr(ao.energy, f)
        assert abs(a - b) <= 1e-9 * max(abs(b), 1.0), (f, a, b)
    for i in range(3):
        assert abs(avg.u[i] - ao.u[i]) <= 1e-9 * max(abs(ao.u[i]), 1.0)
    for i in range(6):
        assert abs(avg.uu[i] - ao.uu[i]) <= 1e-9 * max(abs(ao.uu[i]), 1.0)
        assert abs(avg.strain[i] - ao.strain[i]) <= 1e-9 * max(abs(ao.strain[i]), 1e-6)
    avg_line = (tmp_path / "run.avg").read_text().split()
    assert len(avg_line) == 1 + 3 + 6 + 3 + 6 + 15 + 3 + 6


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
@pytest.mark.parametrize("geom", [dict(L="16 16 16"), dict(L="12 10 8", bulk_or_film="'film'")], ids=["bulk", "film"])
def test_velocity_scaling_steps_match_oracle(fg, prec, geom):
    """velocity_scaling.F:9-103 on the device against the oracle: 8 steps,
    momenta zero outside sum_p and rescaled to 3/2 N k T each step."""
    p = helpers.params(method="'vs'", kelvin="220", **geom)
    o = oracle_lib.Oracle(p)
    u = helpers.seeded_u(p, 41, sigma=0.06)
    q = helpers.seeded_p(p, 41, sigma=0.01)
    o.set_state(u, q)
    eo = o.force()
    with fg.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        eg = ctx.mirror_force_mirror()
        for _ in range(8):
            o.velocity_scaling(eo)
            ctx.velocity_scaling(eg)
        sg = ctx.get_state()
        ke_after = ctx.kinetic_energy_dipo()
    so = o.get_state()
    ref_u, ref_p = A.physical(so["dipoR"], p), A.physical(so["dipoP"], p)
    ru = np.abs(A.physical(sg["dipoR"], p) - ref_u).max() / np.abs(ref_u).max()
    rp = np.abs(A.physical(sg["dipoP"], p) - ref_p).max() / np.abs(ref_p).max()
    ee = helpers.energy_errors(eg, eo, A.POTENTIAL_FIELDS + ["dipo_kinetic"])
    _record(f"vs8[{prec},{'film' if 'bulk_or_film' in geom else 'bulk'}]", dict(u=float(ru), p=float(rp), e=float(max(ee.values()))))
    tol = 1e-10 if prec == A.FG_PREC_FP64 else 2e-5
    assert ru <= tol and rp <= tol and max(ee.values()) <= tol, (ru, rp, ee)
    assert abs(ke_after - p.target_kinetic_energy) <= (1e-12 if prec == A.FG_PREC_FP64 else 1e-6) * p.target_kinetic_energy
