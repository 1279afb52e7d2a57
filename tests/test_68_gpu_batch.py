"""Replica batches (fg_batch_create / fg_batch_step): replicas of different
sizes and methods stepped together in one graph give exactly what each gives
stepped alone (the kernels and their reduction orders are the same)."""
import numpy as np
import pytest

import feram_b200 as fb
import helpers
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu

REPLICAS = [dict(L="16 16 16", kelvin="250"), dict(L="12 10 8", kelvin="300"),
            dict(L="16 16 8", kelvin="200", method="'vs'"), dict(L="8 8 8", kelvin="150", method="'lf'")]


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_batch_equals_replicas_stepped_alone(fg, prec):
    ps = [helpers.params(**r) for r in REPLICAS]
    states = [(helpers.seeded_u(p, 60 + i, sigma=0.05), helpers.seeded_p(p, 60 + i, sigma=0.01))
              for i, p in enumerate(ps)]
    alone = []
    for p, (u, q) in zip(ps, states):
        with fb.Context(p, prec) as ctx:
            ctx.build_tables()
            ctx.set_state(u, q)
            e = ctx.mirror_force_mirror()
            e = ctx.run_steps(6, e)
            st6 = ctx.get_state()
            e10 = ctx.run_steps(10)  # one eight-step graph and two single steps
            alone.append((st6, e, ctx.get_state(), e10))
    with fb.Batch(ps, prec) as b:
        for r, (u, q) in zip(b.replicas, states):
            r.build_tables()
            r.set_state(u, q)
            r.mirror_force_mirror()
        es = b.step(6)
        states6 = [r.get_state() for r in b.replicas]
        es10 = b.step(10)
        for i, (r, p) in enumerate(zip(b.replicas, ps)):
            sa, ea, sa10, ea10 = alone[i]
            for st, s_ref, e_b, e_ref in ((states6[i], sa, es[i], ea), (r.get_state(), sa10, es10[i], ea10)):
                for k in ("dipoR", "dipoP", "dVddi"):
                    assert np.array_equal(A.physical(st[k], p), A.physical(s_ref[k], p)), (i, k)
                assert st["s"] == s_ref["s"] and st["pi"] == s_ref["pi"]
                for f in A.POTENTIAL_FIELDS + ["dipo_kinetic", "total"]:
                    assert getattr(e_b, f) == getattr(e_ref, f), (i, f)


def test_batch_after_replica_site_arrays_change(fg):
    """Uploading site arrays to a replica replaces device buffers that the
    batch's graphs hold: the next fg_batch_step captures them again."""
    ps = [helpers.params(L="16 16 16", kelvin="250"), helpers.params(L="8 8 8", kelvin="300")]
    p0 = ps[0]
    minv = np.zeros((p0.Lz, p0.Ly + p0.padding_y, 2 * (p0.Lx // 2 + 1)))
    minv[:, :p0.Ly, :p0.Lx] = 1.0 / p0.mass_dipo[0]
    minv[3, 4, 5] = 0.0  # one fixed dipole
    states = [(helpers.seeded_u(p, 80 + i, sigma=0.05), helpers.seeded_p(p, 80 + i, sigma=0.01))
              for i, p in enumerate(ps)]
    with fb.Context(p0, A.FG_PREC_MIXED) as ctx:
        ctx.build_tables()
        ctx.set_state(*states[0])
        ctx.mirror_force_mirror()
        ctx.run_steps(3)
        ctx.upload_site_arrays(mass_dipo_inv=minv)
        e_ref = ctx.run_steps(9)
        ref = ctx.get_state()
    with fb.Batch(ps, A.FG_PREC_MIXED) as b:
        for r, st in zip(b.replicas, states):
            r.build_tables()
            r.set_state(*st)
            r.mirror_force_mirror()
        b.step(3)
        b.replicas[0].upload_site_arrays(mass_dipo_inv=minv)
        es = b.step(9)
        got = b.replicas[0].get_state()
    assert np.array_equal(A.physical(got["dipoR"], p0), A.physical(ref["dipoR"], p0))
    assert es[0].total == e_ref.total


def test_batch_rejects_bad_replica(fg):
    good = helpers.params(L="8 8 8")
    bad = A.fg_params.from_buffer_copy(good)
    bad.Lx = 7  # odd Lx with a made N: fg_create refuses it
    with pytest.raises(fb.FeramError, match="replica 1"):
        fb.Batch([good, bad])


def test_batch_epit_field_waves_match_oracle(fg):
    """Config-4-style batch: epitaxial films with their own misfit strain and
    a triangular E_z wave each, the per-step field evaluated on the device
    (fg_set_wave) inside one batch graph; every replica against the oracle's
    molecular_dynamics (molecular-dynamics.F:66-76 with wave_module.F), FP64."""
    import ctypes as C
    import oracle_lib
    strains = (-0.01, 0.0, 0.015)
    periods = (8, 12, 16)
    ps = [helpers.params(L="8 8 8", bulk_or_film="'epit'", epi_strain=str(es), kelvin="280",
                         E_wave_type="'triangular_cos'", external_E_field="0.0 0.0 0.002",
                         n_E_wave_period=str(T), n_thermalize="4", n_average="8")
          for es, T in zip(strains, periods)]
    n = 12
    states = [(helpers.seeded_u(p, 90 + i, sigma=0.05), helpers.seeded_p(p, 90 + i, sigma=0.01))
              for i, p in enumerate(ps)]

    def wave0(p):
        out = (C.c_double * 3)()
        amp = (C.c_double * 3)(*p.external_E_field)
        assert A.lib().fg_wave(p.E_wave_type, 0, p.n_thermalize, p.n_E_wave_period, amp, out) == 0
        return list(out)

    refs = []
    for p, (u, q) in zip(ps, states):
        o = oracle_lib.Oracle(p)
        o.set_state(u, q)
        o.set_uniform_E(wave0(p))
        e = o.force()
        e.dipo_kinetic = o.kinetic_energy_dipo()
        o.md(1, n, 1, e)
        refs.append((o.get_state(), e))
    with fb.Batch(ps, A.FG_PREC_FP64) as b:
        for r, p, (u, q) in zip(b.replicas, ps, states):
            r.build_tables()
            r.set_state(u, q)
            r.set_uniform_E(wave0(p))
            e = r.mirror_force_mirror()
            e.dipo_kinetic = r.kinetic_energy_dipo()
            r.nose_poincare_hamiltonian(e)
            r.set_thermostat(1.0, 0.0, e.H_Nose_Poincare)
            r.set_wave(True, 0)
        es = b.step(n)
        got = [r.get_state() for r in b.replicas]
    for i, (p, (so, eo)) in enumerate(zip(ps, refs)):
        du = np.abs(A.physical(got[i]["dipoR"], p) - A.physical(so["dipoR"], p)).max()
        assert du <= 1e-10, (i, du)
        assert abs(got[i]["s"] - so["s"]) <= 1e-12
        assert np.allclose(got[i]["strain"], so["strain"], rtol=1e-9, atol=1e-14), (i, got[i]["strain"], so["strain"])
        for f in ("total", "dipole_E_field", "unharmonic", "dipo_kinetic"):
            a, c = getattr(es[i], f), getattr(eo, f)
            assert abs(a - c) <= 1e-9 * max(abs(c), 1e-3), (i, f, a, c)


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_grouped_replicas_equal_branches(fg, prec):
    """Replicas of one size (a temperature sweep's points) stepped as one
    launch per kernel give bit for bit what a graph branch per replica
    gives; a replica of another size and a 'vs' replica keep their branches."""
    ps = [helpers.params(L="16 16 16", kelvin=str(400 - 50 * i)) for i in range(4)]
    ps += [helpers.params(L="8 8 8", kelvin="250"), helpers.params(L="16 16 16", kelvin="300", method="'vs'")]
    states = [(helpers.seeded_u(p, 70 + i, sigma=0.05), helpers.seeded_p(p, 70 + i, sigma=0.01))
              for i, p in enumerate(ps)]
    out = {}
    for grouping in (False, True):
        with fb.Batch(ps, prec) as b:
            b.set_grouping(grouping)
            for r, (u, q) in zip(b.replicas, states):
                r.build_tables()
                r.set_state(u, q)
                r.mirror_force_mirror()
            es = b.step(7)
            out[grouping] = ([r.get_state() for r in b.replicas], es, b.groups)
    assert out[False][2] == len(ps) and out[True][2] == 3
    for i, p in enumerate(ps):
        a, c = out[False][0][i], out[True][0][i]
        for k in ("dipoR", "dipoP", "dVddi"):
            assert np.array_equal(A.physical(a[k], p), A.physical(c[k], p)), (i, k)
        assert a["s"] == c["s"] and a["pi"] == c["pi"]
        for f in A.POTENTIAL_FIELDS + ["dipo_kinetic", "total", "H_Nose_Poincare"]:
            assert getattr(out[False][1][i], f) == getattr(out[True][1][i], f), (i, f)


def test_branch_priorities_change_no_bit(fg):
    """Launch priorities on the batch graph's branches (small supercells
    ahead of large ones) only reorder independent kernels: every replica's
    state and energies are the same bit for bit with and without them."""
    ps = [helpers.params(L=f"{n} {n} {n}", kelvin=str(300 - 20 * i)) for i, n in enumerate((8, 16, 16, 24))]
    states = [(helpers.seeded_u(p, 90 + i, sigma=0.05), helpers.seeded_p(p, 90 + i, sigma=0.01))
              for i, p in enumerate(ps)]
    out = {}
    for prio in (False, True):
        with fb.Batch(ps, A.FG_PREC_MIXED) as b:
            b.set_priorities(prio)
            for r, (u, q) in zip(b.replicas, states):
                r.build_tables()
                r.set_state(u, q)
                r.mirror_force_mirror()
            es = b.step(9)
            out[prio] = ([r.get_state() for r in b.replicas], es, b.groups)
    assert out[False][2] == out[True][2] == 3
    for i, p in enumerate(ps):
        a, c = out[False][0][i], out[True][0][i]
        for k in ("dipoR", "dipoP", "dVddi"):
            assert np.array_equal(A.physical(a[k], p), A.physical(c[k], p)), (i, k)
        assert a["s"] == c["s"] and a["pi"] == c["pi"]
        for f in A.POTENTIAL_FIELDS + ["dipo_kinetic", "total", "H_Nose_Poincare"]:
            assert getattr(out[False][1][i], f) == getattr(out[True][1][i], f), (i, f)
