"""What the trained warm-start network gains, and the MD as its referee.

A small network is trained, as warm_start.experiment trains the large one,
on configurations that the GPU MD generates along a 16^3 cooling chain
(moment-matching statistics, then the potential energy through the MD
force).  At a held-out temperature in the ordered phase its proposal, after
the same velocity-scaling settle as a cold start (initialize_dipoR's field),
starts closer to the chained run's equilibrium in the order parameter
|<u>|^2 and in the potential energy than the cold start does.  The
acceptance test (warm_start.accept) takes a run of the same equilibrium and
rejects one of another temperature."""
import ctypes as C

import numpy as np
import pytest

import feram_b200 as fb
import helpers
from feram_b200 import _capi as A
from feram_b200 import warm_start as W

pytestmark = pytest.mark.gpu

L = 16


def _mp(Lw, T, ez, gpa):
    return helpers.params("zzznp.feram", L=f"{Lw} {Lw} {Lw}", kelvin=str(T), GPa=str(gpa), Q_Nose="0.1",
                          init_dipo_avg="0.0 0.0 0.0", init_dipo_dev="0.03 0.03 0.03")


def _equilibrium(T, n_therm=4000, n=3000, every=20):
    """A chained cooling run (400 K down to T) and its trace at T."""
    p = _mp(L, 400.0, 0.0, -5.0)
    with fb.Context(p, A.FG_PREC_MIXED) as ctx:
        ctx.build_tables()
        u, q = A.real_field(p), A.real_field(p)
        assert A.lib().fg_init_dipoR_host(C.byref(p), A.dptr(u), A.dptr(q)) == 0
        W.start_point(ctx, p, u, q)
        for Tc in (400.0, 350.0, 300.0, T):
            ctx.chain_point(Tc, [0.0, 0.0, 0.0])
            ctx.run_steps(n_therm)
        return W.equilibration_trace(ctx, n, every), W.equilibration_trace(ctx, n, every)


def test_trained_net_starts_closer_to_equilibrium_and_is_refereed(fg):
    cond, stats, energies = W.generate_training_set(lambda T, ez, gpa: _mp(L, T, ez, gpa), [(0.0, -5.0)],
                                                    [400.0, 350.0, 300.0, 250.0, 200.0, 150.0],
                                                    n_therm=1500, n_snap=8, snap_every=100)
    assert cond.shape == (48, 5) and stats.shape == (48, W.NSTAT) and energies.shape == (48,)
    T = 225.0  # held out: between the 250 K and 200 K training points, ordered phase
    (Pe, Ve), (Pe2, Ve2) = _equilibrium(T)
    eqP, eqV = float(Pe.mean()), float(Ve.mean())
    probe = W.EnergyProbe(_mp, L)
    try:
        with W.WarmStartNet((L, L, L), batch=8, seed=3) as net:
            hist = W.train(net, cond, stats, steps=800, seed=1, energies=energies, probe=probe, energy_from=400)
            assert np.mean(hist[-20:]) < 0.5 * np.mean(hist[:5])
            net.forward(np.array([[T, 0.0, 0.0, 0.0, -5.0]] * 8), [77 + i for i in range(8)])
            p = _mp(L, T, 0.0, -5.0)
            uw = net.field(0, p)
    finally:
        probe.close()
    first = {}
    with fb.Context(p, A.FG_PREC_MIXED) as ctx:
        ctx.build_tables()
        uc = A.real_field(p)
        assert A.lib().fg_init_dipoR_host(C.byref(p), A.dptr(uc), None) == 0
        for tag, u, q in (("warm", uw, W.maxwell_momenta(p, 5)), ("cold", uc, A.real_field(p))):
            W.start_point(ctx, p, u, q)
            W.settle(ctx, T, [0.0, 0.0, 0.0], 200)
            P, V = W.equilibration_trace(ctx, 400, 20)
            first[tag] = (float(P.mean()), float(V.mean()))
    dw = (abs(first["warm"][0] - eqP), abs(first["warm"][1] - eqV))
    dc = (abs(first["cold"][0] - eqP), abs(first["cold"][1] - eqV))
    assert dw[0] < dc[0] and dw[1] < dc[1], (first, eqP, eqV)
    # the referee: the same equilibrium is accepted, another temperature's is
    # not (blocks of 300 steps: longer than the order parameter's memory)
    assert W.accept(Pe2, Ve2, Pe, Ve, block=15)
    (Ph, Vh), _ = _equilibrium(300.0, n_therm=2000, n=1500)
    assert not W.accept(Ph, Vh, Pe, Ve, block=15)
