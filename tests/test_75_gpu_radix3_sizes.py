"""The 24^3 and 48^3 supercells of the batched sweeps on their compile-time
kernels (transforms of 12, 24 and 48 points: a power-of-two stage and a
radix-3 stage; 4-column z tiles at 24^3 in FP32): force, energies and
Nose-Poincare steps against the oracle, and a grouped batch of them equal
to its replicas stepped alone."""
import ctypes as C

import numpy as np
import pytest

import feram_b200 as fb
import helpers
import oracle_lib
from feram_b200 import _capi as A

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [A.FG_PREC_FP64, A.FG_PREC_MIXED])
@pytest.mark.parametrize("L", [24, 48])
def test_force_and_steps_match_oracle(fg, L, prec):
    p = helpers.params(L=f"{L} {L} {L}", kelvin="250")
    u = helpers.seeded_u(p, 40 + L, sigma=0.08)
    q = helpers.seeded_p(p, 40 + L, sigma=0.01)
    if prec == A.FG_PREC_MIXED:
        u, q = helpers.fp32_config(u), helpers.fp32_config(q)
    o = oracle_lib.Oracle(p)
    o.set_state(u, q)
    eo = o.force()
    eo.dipo_kinetic = o.kinetic_energy_dipo()
    with fb.Context(p, prec) as ctx:
        ctx.build_tables()
        ctx.set_state(u, q)
        eg = ctx.mirror_force_mirror()
        eg.dipo_kinetic = ctx.kinetic_energy_dipo()
        fmax, frms = helpers.force_error(ctx.get_state()["dVddi"], o.get_state()["dVddi"], p)
        ee = helpers.energy_errors(eg, eo)
        ftol, etol = (1e-12, 1e-12) if prec == A.FG_PREC_FP64 else (1e-6, 1e-5)
        assert fmax <= ftol and frms <= ftol and max(ee.values()) <= etol, (fmax, frms, ee)
        o.set_state(None, None, 1.0, 0.0, 0.0)
        h = o.L.oracle_nose_poincare_hamiltonian(o.h, C.byref(eo))
        o.set_state(None, None, 1.0, 0.0, h)
        ctx.set_thermostat(1.0, 0.0, h)
        for _ in range(4):
            o.nose_poincare(eo)
            ctx.nose_poincare(eg)
        sg, so = ctx.get_state(), o.get_state()
    ru = np.abs(A.physical(sg["dipoR"], p) - A.physical(so["dipoR"], p)).max() / np.abs(A.physical(so["dipoR"], p)).max()
    tol = 1e-10 if prec == A.FG_PREC_FP64 else 2e-5
    assert ru <= tol and abs(sg["s"] - so["s"]) <= tol, (ru, sg["s"], so["s"])


def test_grouped_batch_of_24_and_48_equals_replicas_alone(fg):
    ps = [helpers.params(L="24 24 24", kelvin="300"), helpers.params(L="24 24 24", kelvin="250"),
          helpers.params(L="48 48 48", kelvin="200"), helpers.params(L="48 48 48", kelvin="150")]
    states = [(helpers.seeded_u(p, 70 + i, sigma=0.05), helpers.seeded_p(p, 70 + i, sigma=0.01))
              for i, p in enumerate(ps)]
    alone = []
    for p, (u, q) in zip(ps, states):
        with fb.Context(p, A.FG_PREC_MIXED) as ctx:
            ctx.build_tables()
            ctx.set_state(u, q)
            ctx.mirror_force_mirror()
            ctx.run_steps(9)
            alone.append(ctx.get_state())
    with fb.Batch(ps, A.FG_PREC_MIXED) as b:
        for r, (u, q) in zip(b.replicas, states):
            r.build_tables()
            r.set_state(u, q)
            r.mirror_force_mirror()
        b.step(9)
        assert b.groups == 2
        for i, (r, p) in enumerate(zip(b.replicas, ps)):
            st = r.get_state()
            for k in ("dipoR", "dipoP"):
                assert np.array_equal(A.physical(st[k], p), A.physical(alone[i][k], p)), (i, k)
            assert st["s"] == alone[i]["s"]
