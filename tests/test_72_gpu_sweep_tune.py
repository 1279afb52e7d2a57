"""Launch plans and their autotuner (fg_tune, fg_batch_tune, fg_set_plan,
wisdom), the device sample series (fg_sample) and sweep points
(fg_run_point, fg_batch_run_point).

The reference plans its FFTs with FFTW_MEASURE (coord_module.F:155-377) and
reads saved wisdom at start-up (feram_common.F:56-69); a plan changes the
order of floating-point work, not the Hamiltonian, so every plan must give
the oracle's force, and tuning must leave the dynamical state as it was.
A sweep point is a point of the reference's cooling scripts (cooling.sh:64-69
chaining n_thermalize + n_average runs); its samples are the per-step
quantities of add_to_Average (average_module.F:75-128)."""
import ctypes as C

import numpy as np
import pytest

import feram_b200 as fb
import helpers
import oracle_lib
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _no_wisdom(fg):
    fb.wisdom_forget()
    yield
    fb.wisdom_forget()


def _zcw_candidates(p, prec):
    cap = 8 if prec == A.FG_PREC_MIXED else 4
    out, last = [], None
    w = cap
    while w >= 1 and len(out) < 3:
        cw = w
        while cw > 1 and (p.Lx // 2) % cw:
            cw //= 2
        if cw != last:
            out.append(w)
        last = cw
        w //= 2
    return out


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
@pytest.mark.parametrize("L", ["16 16 16", "24 12 8"])
def test_every_plan_gives_the_oracle_force(fg, prec, L):
    """Each z-tile width and streaming grid the tuner may pick: force and
    energies against the oracle (FP64 1e-12; mixed, on FP32-exact
    configurations: force 1e-6, energies 1e-5)."""
    p = helpers.params(L=L, kelvin="250")
    u = helpers.seeded_u(p, 17, sigma=0.06)
    uo = helpers.fp32_config(u) if prec == A.FG_PREC_MIXED else u
    o = oracle_lib.Oracle(p)
    o.set_state(uo, None)
    eo = o.force()
    Fo = o.get_state()["dVddi"]
    seen = set()
    with fb.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(uo)
        for z in _zcw_candidates(p, prec):
            for w in (1, 2, 0):
                ctx.set_plan(z, w)
                cw, waves, gkd, gas = ctx.plan
                assert waves == w and cw <= max(z, 1) and (p.Lx // 2) % cw == 0
                seen.add(cw)
                eg = ctx.mirror_force_mirror()
                fmax, _ = helpers.force_error(ctx.get_state()["dVddi"], Fo, p)
                ee = helpers.energy_errors(eg, eo)
                ftol, etol = (1e-12, 1e-12) if prec == A.FG_PREC_FP64 else (1e-6, 1e-5)
                assert fmax <= ftol and max(ee.values()) <= etol, (z, w, fmax, ee)
    assert len(seen) >= 2


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_tune_restores_the_state_and_feeds_wisdom(fg, prec):
    p = helpers.params(L="16 16 16", kelvin="250")
    u, q = helpers.seeded_u(p, 5, sigma=0.05), helpers.seeded_p(p, 5, sigma=0.01)
    with fb.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        e0 = ctx.mirror_force_mirror()
        ctx.run_steps(3)
        before = ctx.get_state()
        cw, waves, ms = ctx.tune(steps=8)
        assert ms > 0.0 and ctx.plan[:2] == (cw, waves)
        after = ctx.get_state()
        for k in ("dipoR", "dipoP"):
            assert np.array_equal(A.physical(after[k], p), A.physical(before[k], p)), k
        for k in ("s", "pi", "H0"):
            assert after[k] == before[k], k
        assert np.array_equal(after["strain"], before["strain"])
        # the tuned context steps on as the untuned one does (same Hamiltonian)
        e1 = ctx.run_steps(4)
    with fb.Context(p, prec) as ref:
        assert ref.plan[:2] == (cw, waves)  # the wisdom is applied at creation
        ref.set_plan(0, 1)
        ref.build_tables()
        ref.set_state(u, q)
        ref.mirror_force_mirror()
        ref.run_steps(3)
        e2 = ref.run_steps(4)
    tol = 1e-11 if prec == A.FG_PREC_FP64 else 1e-5
    assert abs(e1.total - e2.total) <= tol * abs(e2.total), (e1.total, e2.total)
    text = fb.wisdom_export()
    mode_prec = "solo " + ("mixed" if prec == A.FG_PREC_MIXED else "fp64")
    assert any(line.startswith(mode_prec + " 16 16 16 9 ") for line in text.splitlines()), text
    assert e0.short_range != 0.0


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_samples_are_the_average_module_quantities(fg, prec):
    """A sample row holds what fg_average_accumulate adds for the same state
    (the same device sums), and the series empties on reading."""
    p = helpers.params(L="12 10 8", kelvin="300")
    u, q = helpers.seeded_u(p, 9, sigma=0.05, avg=0.02), helpers.seeded_p(p, 9, sigma=0.01)
    with fb.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        ctx.mirror_force_mirror()
        rows = []
        for _ in range(3):
            e = ctx.run_steps(5)
            ctx.sample()
            avg = A.fg_average()
            ctx.average_accumulate(e, avg)
            st = ctx.get_state()
            rows.append((avg, e, st))
        S = ctx.samples()
        assert S.shape == (3, A.FG_SAMPLE_COLS)
        assert ctx.samples().shape == (0, A.FG_SAMPLE_COLS)
    for r, (avg, e, st) in zip(S, rows):
        assert np.array_equal(r[0:3], np.array(avg.u[:])), (r[0:3], avg.u[:])
        assert np.array_equal(r[3:6], np.array(avg.p[:]))
        V = sum(getattr(e, f) for f in A.POTENTIAL_FIELDS)
        assert abs(r[6] - V) <= 1e-12 * abs(V)
        assert abs(r[7] - e.dipo_kinetic / st["s"] ** 2) <= 1e-12 * abs(r[7])
        assert r[8] == st["s"] and r[9] == st["pi"]
        assert np.array_equal(r[10:16], st["strain"])


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_batch_sweep_point_equals_points_run_alone(fg, prec):
    """fg_batch_run_point (grouped and single branches) against fg_run_point
    of each replica alone: the same samples and states bit for bit, over two
    chained points."""
    specs = [("16 16 16", 300.0, 250.0), ("16 16 16", 280.0, 230.0), ("12 10 8", 260.0, 210.0)]
    ps = [helpers.params(L=L, kelvin=str(T0)) for L, T0, _ in specs]
    states = [(helpers.seeded_u(p, 30 + i, sigma=0.05), helpers.seeded_p(p, 30 + i, sigma=0.01))
              for i, p in enumerate(ps)]
    E = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.0], [0.0, 0.0, 5e-4]])  # equal fields keep 0, 1 grouped
    alone = []
    for i, (p, (u, q)) in enumerate(zip(ps, states)):
        with fb.Context(p, prec) as ctx:
            ctx.build_tables()
            ctx.set_state(u, q)
            ctx.mirror_force_mirror()
            ctx.run_point(specs[i][1], 12, 30, 10, E[i])
            s1 = ctx.samples()
            ctx.run_point(specs[i][2], 8, 20, 5, E[i])
            alone.append((s1, ctx.samples(), ctx.get_state()))
    with fb.Batch(ps, prec) as b:
        for r, (u, q) in zip(b.replicas, states):
            r.build_tables()
            r.set_state(u, q)
            r.mirror_force_mirror()
        b.run_point([s[1] for s in specs], 12, 30, 10, E)
        s1 = b.samples()
        b.run_point([s[2] for s in specs], 8, 20, 5, E)
        s2 = b.samples()
        assert b.groups == 2
        for i, r in enumerate(b.replicas):
            a1, a2, ast = alone[i]
            assert s1[i].shape == (3, A.FG_SAMPLE_COLS) and s2[i].shape == (4, A.FG_SAMPLE_COLS)
            assert np.array_equal(s1[i], a1), i
            assert np.array_equal(s2[i], a2), i
            st = r.get_state()
            assert np.array_equal(A.physical(st["dipoR"], ps[i]), A.physical(ast["dipoR"], ps[i])), i
            assert st["s"] == ast["s"] and r.p.kelvin == specs[i][2]


def test_batch_tune_restores_states_and_plans_by_supercell(fg):
    ps = [helpers.params(L="16 16 16", kelvin="300"), helpers.params(L="16 16 16", kelvin="250"),
          helpers.params(L="24 24 24", kelvin="200")]
    states = [(helpers.seeded_u(p, 50 + i, sigma=0.05), helpers.seeded_p(p, 50 + i, sigma=0.01))
              for i, p in enumerate(ps)]
    with fb.Batch(ps, A.FG_PREC_MIXED) as b:
        for r, (u, q) in zip(b.replicas, states):
            r.build_tables()
            r.set_state(u, q)
            r.mirror_force_mirror()
        b.step(2)
        before = [r.get_state() for r in b.replicas]
        t0, t1 = b.tune(steps=4)
        assert 0.0 < t1 <= t0
        for r, s, p in zip(b.replicas, before, ps):
            st = r.get_state()
            assert np.array_equal(A.physical(st["dipoR"], p), A.physical(s["dipoR"], p))
            assert st["s"] == s["s"] and st["pi"] == s["pi"]
        assert b.replicas[0].plan == b.replicas[1].plan  # one plan per supercell
        plans = [r.plan[:2] for r in b.replicas]
        b.step(3)
        assert b.groups == 2
    lines = fb.wisdom_export().splitlines()
    assert any(line.startswith("batch mixed 16 16 16 9 ") for line in lines), lines
    assert any(line.startswith("batch mixed 24 24 24 9 ") for line in lines), lines
    with fb.Batch(ps, A.FG_PREC_MIXED) as b2:  # batch wisdom at creation
        assert [r.plan[:2] for r in b2.replicas] == plans


def test_sample_series_overflow_is_an_error(fg):
    p = helpers.params(L="8 8 8", kelvin="300")
    with fb.Context(p, A.FG_PREC_MIXED) as ctx:
        ctx.build_tables()
        ctx.set_state(helpers.seeded_u(p, 1, sigma=0.05))
        ctx.mirror_force_mirror()
        with pytest.raises(fb.FeramError) as ei:
            ctx.run_point(300.0, 0, (A.FG_SAMPLE_CAP + 1) * 2, 2)
        assert "overflow" in str(ei.value)
        ctx.run_point(300.0, 0, 40, 2)
        assert ctx.samples().shape == (20, A.FG_SAMPLE_COLS)


def test_wisdom_measure_and_the_driver_reads_gpu_wisdom(fg, tmp_path):
    """fg_wisdom_measure tunes a supercell as feram_fftw_wisdom measures FFTW
    plans; fg_feram_run imports a gpu_wisdom file beside its input before it
    makes the context (feram_common.F:56-69) and says so in the .log; a
    malformed file leaves the default plans and is reported."""
    text = fb.wisdom_measure(helpers.params(L="8 8 8"), 8, A.FG_PREC_FP64)
    lines = [ln for ln in text.splitlines() if ln.startswith("solo fp64 8 8 8 ")]
    assert len(lines) == 1, text
    fb.wisdom_forget()
    deck = helpers.deck(L="8 8 8", n_thermalize="4", n_average="4")
    (tmp_path / "run.feram").write_text(deck)
    (tmp_path / "gpu_wisdom").write_text(text)
    avg_w, _ = fg.feram_run(str(tmp_path / "run.feram"), A.FG_PREC_FP64)
    log = (tmp_path / "run.log").read_text().splitlines()
    assert log[0].startswith("GPU_WISDOM Successfully imported"), log[0]
    assert any(ln.startswith("solo fp64 8 8 8 ") for ln in fb.wisdom_export().splitlines())
    fb.wisdom_forget()
    (tmp_path / "gpu_wisdom").write_text("not wisdom\n")
    avg_d, _ = fg.feram_run(str(tmp_path / "run.feram"), A.FG_PREC_FP64)
    assert (tmp_path / "run.log").read_text().splitlines()[0].startswith("GPU_WISDOM Failed")
    assert avg_w.n_steps == avg_d.n_steps
    # the plan changes the order of the energy sums only
    assert abs(avg_w.energy.total - avg_d.energy.total) <= 1e-10 * abs(avg_d.energy.total)
