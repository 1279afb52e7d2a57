"""Per-site arrays (fg_upload_site_arrays): two relaxor species with their
own on-site polynomials and masses (read_relaxor.F, dVddi-unharmonic.F),
fixed defect dipoles (read_defects_u.F: zero inverse mass, out of sum_p) and
a local field (initialize_E_field.F:14-45), against the oracle."""
import ctypes as C

import numpy as np
import pytest

import feram_b200 as fb
import helpers
import oracle_lib
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu

# per-species tags take RELAXOR_MAX = 3 values (param_module.F:227-236)
TWO_SPECIES = dict(P_kappa2="5.502 4.61 4.61", P_alpha="110.4 98.2 98.2", P_gamma="-163.1 -151.0 -151.0",
                   mass_amu="39.0 47.5 47.5", Z_star="9.956 9.956 9.956")


def _sites(p, seed):
    rng = np.random.default_rng(seed)
    shape = (p.Lz, p.Ly + p.padding_y, 2 * (p.Lx // 2 + 1))
    relaxor = np.ones(shape, dtype=np.int32)
    relaxor[:, :p.Ly, :p.Lx] = rng.integers(1, 3, size=(p.Lz, p.Ly, p.Lx))
    minv = np.zeros(shape)
    minv[:, :p.Ly, :p.Lx] = 1.0 / np.array([p.mass_dipo[0], p.mass_dipo[1]])[relaxor[:, :p.Ly, :p.Lx] - 1]
    sum_p = np.zeros(shape, dtype=np.int32)
    sum_p[:, :p.Ly, :p.Lx] = 1
    defects = [(1, 2, 3), (5, 0, 7), (7, 7, 0), (3, 3, 3)]
    for x, y, z in defects:
        minv[z, y, x] = 0.0
        sum_p[z, y, x] = 0
    eloc = A.real_field(p)
    A.physical(eloc, p)[...] = rng.standard_normal((p.Lz, p.Ly, p.Lx, 3)) * 2e-3
    return relaxor, minv, sum_p, eloc, defects


def _state(p, seed, defects):
    u = helpers.seeded_u(p, seed, sigma=0.06)
    q = helpers.seeded_p(p, seed, sigma=0.01)
    for x, y, z in defects:
        A.physical(u, p)[z, y, x] = (0.05, -0.02, 0.08)
        A.physical(q, p)[z, y, x] = 0.0
    return u, q


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_site_arrays_force_and_nose_poincare_match_oracle(fg, prec):
    p = helpers.params(L="8 8 8", kelvin="260", **TWO_SPECIES)
    relaxor, minv, sum_p, eloc, defects = _sites(p, 5)
    u, q = _state(p, 5, defects)
    o = oracle_lib.Oracle(p)
    o.set_sites(relaxor=relaxor, mass_dipo_inv=minv, sum_p=sum_p, E_field_local=eloc)
    o.set_uniform_E([0.0, 0.0, 0.0005])
    o.set_state(u, q)
    eo = o.force()
    eo.dipo_kinetic = o.kinetic_energy_dipo()
    with fb.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.upload_site_arrays(relaxor=relaxor, mass_dipo_inv=minv, sum_p=sum_p, E_field_local=eloc)
        ctx.set_uniform_E([0.0, 0.0, 0.0005])
        ctx.set_state(u, q)
        eg = ctx.mirror_force_mirror()
        eg.dipo_kinetic = ctx.kinetic_energy_dipo()
        fmax, _ = helpers.force_error(ctx.get_state()["dVddi"], o.get_state()["dVddi"], p)
        ee = helpers.energy_errors(eg, eo, A.POTENTIAL_FIELDS + ["dipo_kinetic"])
        tol = 1e-11 if prec == A.FG_PREC_FP64 else 1e-5
        assert fmax <= tol and max(ee.values()) <= tol, (fmax, ee)
        assert eg.dipole_E_field != 0.0
        # Nose-Poincare steps with the per-site masses and masks
        o.set_state(None, None, 1.0, 0.0, 0.0)
        h = o.L.oracle_nose_poincare_hamiltonian(o.h, C.byref(eo))
        o.set_state(None, None, 1.0, 0.0, h)
        ctx.set_thermostat(1.0, 0.0, h)
        for _ in range(6):
            o.nose_poincare(eo)
            ctx.nose_poincare(eg)
        sg, so = ctx.get_state(), o.get_state()
    ug, uo = A.physical(sg["dipoR"], p), A.physical(so["dipoR"], p)
    for x, y, z in defects:  # fixed dipoles stay put
        assert np.allclose(ug[z, y, x], (0.05, -0.02, 0.08), rtol=0, atol=1e-7)
        assert np.allclose(uo[z, y, x], (0.05, -0.02, 0.08), rtol=0, atol=0)
    ru = np.abs(ug - uo).max() / np.abs(uo).max()
    tol = 1e-10 if prec == A.FG_PREC_FP64 else 2e-5
    assert ru <= tol and abs(sg["s"] - so["s"]) <= tol, (ru, sg["s"], so["s"])


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_species_with_different_zstar_match_oracle(fg, prec):
    """Species with their own Z* (read_relaxor.F:35): the device derives
    Z*(R) from the species and transforms Z* u on its own; short- and
    long-range parts as dVddi-dipole-dipole.F:20-60, the field term with
    Z*(R) (mirror_force_mirror.F:42-50)."""
    p = helpers.params(L="8 8 8", kelvin="260", **dict(TWO_SPECIES, Z_star="9.956 7.2 7.2"))
    relaxor, minv, sum_p, eloc, defects = _sites(p, 6)
    zs = np.zeros(relaxor.shape)
    zs[:, :p.Ly, :p.Lx] = np.array(p.Z_star[:3])[relaxor[:, :p.Ly, :p.Lx] - 1]
    u, q = _state(p, 6, defects)
    o = oracle_lib.Oracle(p)
    o.set_sites(Z_starR=zs, relaxor=relaxor, mass_dipo_inv=minv, sum_p=sum_p, E_field_local=eloc)
    o.set_uniform_E([0.0, 0.0005, 0.0])
    o.set_state(u, q)
    eo = o.force()
    with fb.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.upload_site_arrays(relaxor=relaxor, mass_dipo_inv=minv, sum_p=sum_p, E_field_local=eloc)
        ctx.set_uniform_E([0.0, 0.0005, 0.0])
        ctx.set_state(u, q)
        eg = ctx.mirror_force_mirror()
        fmax, _ = helpers.force_error(ctx.get_state()["dVddi"], o.get_state()["dVddi"], p)
        ee = helpers.energy_errors(eg, eo, A.POTENTIAL_FIELDS)
        tol = 1e-11 if prec == A.FG_PREC_FP64 else 1e-5
        assert fmax <= tol and max(ee.values()) <= tol, (fmax, ee)
        # the long-range energy differs from the uniform-Z* value
        o2 = oracle_lib.Oracle(p)
        o2.set_state(u, q)
        assert abs(o2.force().long_range - eo.long_range) > 1e-3 * abs(eo.long_range)
        o.set_state(None, None, 1.0, 0.0, 0.0)
        h = o.L.oracle_nose_poincare_hamiltonian(o.h, C.byref(eo))
        o.set_state(None, None, 1.0, 0.0, h)
        ctx.set_thermostat(1.0, 0.0, h)
        for _ in range(5):
            o.nose_poincare(eo)
            ctx.nose_poincare(eg)
        sg, so = ctx.get_state(), o.get_state()
    ug, uo = A.physical(sg["dipoR"], p), A.physical(so["dipoR"], p)
    ru = np.abs(ug - uo).max() / np.abs(uo).max()
    tol = 1e-10 if prec == A.FG_PREC_FP64 else 2e-5
    assert ru <= tol and abs(sg["s"] - so["s"]) <= tol, (ru, sg["s"], so["s"])


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
def test_per_site_zstar_array_with_acoustic_leapfrog(fg, prec):
    """An arbitrary Z*(R) array with acoustic-displacement leapfrog: fifteen
    force components (u, u u, acouR, Z* u) through the transforms."""
    p = helpers.params("zzzlf.feram", L="12 10 8", kelvin="200")
    assert p.mass_acou[0] > 0.0
    rng = np.random.default_rng(9)
    shape = (p.Lz, p.Ly + p.padding_y, 2 * (p.Lx // 2 + 1))
    zs = np.zeros(shape)
    zs[:, :p.Ly, :p.Lx] = p.Z_star[0] * (1.0 + 0.2 * rng.standard_normal((p.Lz, p.Ly, p.Lx)))
    u = helpers.seeded_u(p, 21, sigma=0.06, avg=0.05)
    q = helpers.seeded_p(p, 21, sigma=0.01)
    ar = helpers.seeded_u(p, 98, sigma=0.003)
    ap = helpers.seeded_u(p, 99, sigma=0.004)
    o = oracle_lib.Oracle(p)
    o.set_sites(Z_starR=zs)
    o.set_uniform_E([0.0004, 0.0, 0.0])
    o.set_state(u, q)
    o.set_acou(ar, ap)
    eo = A.fg_energy()
    with fb.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.upload_site_arrays(Z_starR=zs)
        ctx.set_uniform_E([0.0004, 0.0, 0.0])
        ctx.set_state(u, q)
        ctx.set_acou(ar, ap)
        eg = A.fg_energy()
        for step in range(0, 6):
            o.leapfrog(eo, step)
            ctx.leapfrog(eg, step)
        sg, so = ctx.get_state(), o.get_state()
        ag, ao = ctx.get_acou(), o.get_acou()
    tol = 1e-10 if prec == A.FG_PREC_FP64 else 2e-5
    for a, b in ((sg["dipoR"], so["dipoR"]), (sg["dVddi"], so["dVddi"]), (ag["acouR"], ao["acouR"])):
        a, b = A.physical(a, p), A.physical(b, p)
        assert np.abs(a - b).max() / np.abs(b).max() <= tol
    ee = helpers.energy_errors(eg, eo, A.POTENTIAL_FIELDS + ["dipo_kinetic", "acou_kinetic"])
    assert max(ee.values()) <= tol, ee


def test_failed_site_upload_leaves_no_stale_graph(fg):
    """A site upload that replaces buffers and then fails (here: a per-site
    Z* whose 12-component z tiles do not fit in shared memory at Lz = 1280,
    FP64, while the plain 9-component tiles do) must not leave a step graph
    that holds the freed buffers: the next step is refused with an error
    instead of replaying the graph."""
    p = helpers.params(L="4 4 1280", Q_Nose="1.0", Z_star="9.956 7.0 7.0", **{
        k: v for k, v in TWO_SPECIES.items() if k != "Z_star"})
    u = helpers.seeded_u(p, 3, sigma=0.05)
    shape = (p.Lz, p.Ly + p.padding_y, 2 * (p.Lx // 2 + 1))
    relaxor = np.ones(shape, dtype=np.int32)
    relaxor[:, :p.Ly, :p.Lx] = 1
    relaxor[::2, :p.Ly, :p.Lx] = 2  # species 2 has its own Z*: per-site Z* path
    with fb.Context(p, A.FG_PREC_FP64) as ctx:
        ctx.build_tables()
        ctx.set_state(u)
        e = ctx.mirror_force_mirror()
        e.dipo_kinetic = ctx.kinetic_energy_dipo()
        ctx.nose_poincare(e)  # captures the step graph with the current tables
        with pytest.raises(fb.FeramError) as ei:
            ctx.upload_site_arrays(relaxor=relaxor)
        assert ei.value.code == A.FG_ERR_UNSUPPORTED, ei.value
        with pytest.raises(fb.FeramError) as ei:
            ctx.nose_poincare(e)
        assert "destroy this context" in str(ei.value)
