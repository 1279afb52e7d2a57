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
            alone.append((ctx.get_state(), e))
    with fb.Batch(ps, prec) as b:
        for r, (u, q) in zip(b.replicas, states):
            r.build_tables()
            r.set_state(u, q)
            r.mirror_force_mirror()
        es = b.step(6)
        for i, (r, p) in enumerate(zip(b.replicas, ps)):
            st = r.get_state()
            sa, ea = alone[i]
            for k in ("dipoR", "dipoP", "dVddi"):
                assert np.array_equal(A.physical(st[k], p), A.physical(sa[k], p)), (i, k)
            assert st["s"] == sa["s"] and st["pi"] == sa["pi"]
            for f in A.POTENTIAL_FIELDS + ["dipo_kinetic", "total"]:
                assert getattr(es[i], f) == getattr(ea, f), (i, f)


def test_batch_rejects_bad_replica(fg):
    good = helpers.params(L="8 8 8")
    bad = A.fg_params.from_buffer_copy(good)
    bad.Lx = 7  # odd Lx with a made N: fg_create refuses it
    with pytest.raises(fb.FeramError, match="replica 1"):
        fb.Batch([good, bad])
