"""Learned warm start for sweep points (no counterpart in the reference).

The reference starts every point of a temperature or field sweep from the
previous point's final state (its sweep scripts link the last .coord as the
next .restart, e.g. 03example-BaTiO3-bulk-phase-transition/16x16x16-40000-
10000/cooling.sh:64-69; here fg_chain_point does that on the device).  This
module trains a small periodic 3D convolutional network on configurations
the MD generates, so that it proposes a field u(R) for a new (T, E, p) point
that starts closer to equilibrium; the MD then judges the proposal: a warm
start whose averages fall outside the statistical error of a plain run is
rejected and the point falls back to the chained start.

Everything here is orchestration of the C-ABI (fg_ws_* for the network, whose
convolutions and their gradients run on the tensor cores; the MD calls for
the data); no arithmetic of the model runs in Python except the site
statistics of the training targets, which restate those of the device.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _capi as A
from ._capi import FG_PREC_MIXED

NSTAT = 7
STAT_NAMES = ("m.e", "|m|", "(sum m_a^4)^1/4", "<|u|^2>", "<sum u_a^4>", "C_long", "C_trans")
E_SCALE = 0.001  # V/A: 100 kV/cm


def site_stats(u: np.ndarray, E) -> np.ndarray:
    """The seven statistics of a configuration u (Lz, Ly, Lx, 3) at field E:
    m.e, |m|, (sum_a m_a^4)^(1/4) (m = <u>, e = E / 0.001 V/A; floors 1e-8
    and 1e-16 under the roots), <|u|^2>, <sum_a u_a^4>,
    <sum_a u_a(R) u_a(R + a)>, <sum_a sum_b!=a u_a(R) u_a(R + b)>."""
    u = np.asarray(u, dtype=np.float64)
    m = u.reshape(-1, 3).mean(axis=0)
    e = np.asarray(E, dtype=np.float64) / E_SCALE
    ax = {0: 2, 1: 1, 2: 0}  # component a -> array axis of direction a (z, y, x order)
    c_long = sum((u[..., a] * np.roll(u[..., a], -1, axis=ax[a])).mean() for a in range(3))
    c_tr = sum((u[..., a] * np.roll(u[..., a], -1, axis=ax[b])).mean() for a in range(3) for b in range(3) if b != a)
    return np.array([m @ e, np.sqrt(m @ m + 1e-8), np.sqrt(np.sqrt((m ** 4).sum() + 1e-16)), (u ** 2).sum(-1).mean(),
                     (u ** 4).sum(-1).mean(), c_long, c_tr])


class WarmStartNet:
    """fg_ws: the network of `batch` samples of an Lx x Ly x Lz supercell."""

    def __init__(self, L, batch: int = 8, seed: int = 1):
        self.L = tuple(L)
        self.batch = batch
        self._h = C.c_void_p()
        rc = A.lib().fg_ws_create(L[0], L[1], L[2], batch, seed, C.byref(self._h))
        if rc:
            msg = A.lib().fg_ws_last_error(self._h).decode()
            self.close()
            raise RuntimeError(f"fg_ws_create [{rc}]: {msg}")

    def _check(self, rc):
        if rc:
            raise RuntimeError(f"fg_ws [{rc}]: {A.lib().fg_ws_last_error(self._h).decode()}")

    @staticmethod
    def _f32(a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        return a, a.ctypes.data_as(C.POINTER(C.c_float))

    def _inputs(self, cond, seeds):
        cond, cp = self._f32(np.asarray(cond).reshape(self.batch, 5))
        sd = (C.c_ulonglong * self.batch)(*[int(x) for x in seeds])
        return cond, cp, sd

    def forward(self, cond, seeds) -> np.ndarray:
        """Statistics [batch][7] of the generated fields."""
        keep, cp, sd = self._inputs(cond, seeds)
        S = np.zeros((self.batch, NSTAT), dtype=np.float32)
        self._check(A.lib().fg_ws_forward(self._h, cp, sd, S.ctypes.data_as(C.POINTER(C.c_float))))
        return S

    def backward(self, cond, seeds, target, weights, dLdu=None) -> float:
        """Loss and gradients (fg_ws_backward); with dLdu [batch][N][3] a
        further gradient on the generated u (fg_ws_backward_du)."""
        keep, cp, sd = self._inputs(cond, seeds)
        t, tp = self._f32(np.asarray(target).reshape(self.batch, NSTAT))
        w, wp = self._f32(weights)
        loss = C.c_float()
        if dLdu is None:
            self._check(A.lib().fg_ws_backward(self._h, cp, sd, tp, wp, C.byref(loss)))
        else:
            n = self.batch * self.L[0] * self.L[1] * self.L[2]
            g, gp = self._f32(np.asarray(dLdu).reshape(n, 3))
            self._check(A.lib().fg_ws_backward_du(self._h, cp, sd, tp, wp, gp, C.byref(loss)))
        return float(loss.value)

    def adam(self, lr: float):
        self._check(A.lib().fg_ws_adam(self._h, lr))

    def layer(self, l: int):
        co, ci = C.c_int(), C.c_int()
        self._check(A.lib().fg_ws_layer_shape(self._h, l, C.byref(co), C.byref(ci)))
        w = np.zeros((co.value, 27, ci.value), dtype=np.float32)
        b = np.zeros(co.value, dtype=np.float32)
        dw, db = np.zeros_like(w), np.zeros_like(b)
        f = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        self._check(A.lib().fg_ws_get_layer(self._h, l, f(w), f(b), f(dw), f(db)))
        return w, b, dw, db

    def set_layer(self, l: int, w, b):
        w, wp = self._f32(w)
        b, bp = self._f32(b)
        self._check(A.lib().fg_ws_set_layer(self._h, l, wp, bp))

    def io(self):
        """(layer-1 input [B*N][16], generated u [B*N][3]) of the last forward."""
        n = self.batch * self.L[0] * self.L[1] * self.L[2]
        x = np.zeros((n, 16), dtype=np.float32)
        u = np.zeros((n, 3), dtype=np.float32)
        f = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        self._check(A.lib().fg_ws_get_io(self._h, f(x), f(u)))
        return x, u

    def field(self, b: int, p) -> np.ndarray:
        """Sample b of the last forward as a padded dipoR array for p."""
        u = A.real_field(p)
        self._check(A.lib().fg_ws_field(self._h, b, p.padding_y, A.dptr(u)))
        return u

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            A.lib().fg_ws_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def maxwell_momenta(p, seed: int) -> np.ndarray:
    """Momenta drawn from the Maxwell-Boltzmann distribution at p.kelvin
    (p_a ~ N(0, sqrt(m k T)) per site and component), padded layout."""
    rng = np.random.default_rng(seed)
    q = A.real_field(p)
    sd = np.sqrt(p.mass_dipo[0] * p.temperature_eV)
    A.physical(q, p)[...] = rng.standard_normal((p.Lz, p.Ly, p.Lx, 3)) * sd
    return q


def start_point(ctx, p, u, q) -> "A.fg_energy":
    """initialize_dipoR's tail and molecular-dynamics.F:52-55 for a given
    (u, p): force, s = 1, pi = 0, H0 from the state."""
    ctx.set_state(u, q, 1.0, 0.0, 0.0)
    ctx.set_uniform_E([p.external_E_field[0], p.external_E_field[1], p.external_E_field[2]])
    e = ctx.mirror_force_mirror()
    e.dipo_kinetic = ctx.kinetic_energy_dipo()
    ctx.nose_poincare_hamiltonian(e)
    ctx.set_thermostat(1.0, 0.0, e.H_Nose_Poincare)
    return e


def potential(e) -> float:
    return sum(getattr(e, f) for f in A.POTENTIAL_FIELDS)


def generate_training_set(make_params, chains, temps, n_therm=3000, n_snap=14, snap_every=100,
                          precision=FG_PREC_MIXED):
    """Configurations generated by the MD: one cooling chain per (E_z, GPa)
    in `chains`, each through `temps` (descending), every point started from
    the previous one on the device (fg_chain_point), thermalised n_therm
    steps, then n_snap snapshots snap_every steps apart.  All chains step
    together as one replica batch.  Returns (cond [n][5], stats [n][7],
    potential energy per site [n])."""
    import feram_b200 as fb
    ps = [make_params(temps[0], Ez, gpa) for Ez, gpa in chains]
    conds, stats, energies = [], [], []
    with fb.Batch(ps, precision) as b:
        for i, (r, p) in enumerate(zip(b.replicas, ps)):
            r.build_tables()
            u = A.real_field(p)
            q = A.real_field(p)
            assert A.lib().fg_init_dipoR_host(C.byref(p), A.dptr(u), A.dptr(q)) == 0
            start_point(r, p, u, q)
        for k, T in enumerate(temps):
            if k > 0:
                for r, (Ez, gpa) in zip(b.replicas, chains):
                    r.chain_point(T, [0.0, 0.0, Ez])
            b.step(n_therm)
            for _ in range(n_snap):
                es = b.step(snap_every)
                for r, e, (Ez, gpa) in zip(b.replicas, es, chains):
                    u = A.physical(r.get_state()["dipoR"], r.p)
                    conds.append([T, 0.0, 0.0, Ez, gpa])
                    stats.append(site_stats(u, [0.0, 0.0, Ez]))
                    energies.append(potential(e) / r.p.N)
    return (np.array(conds, dtype=np.float64), np.array(stats, dtype=np.float64),
            np.array(energies, dtype=np.float64))


class EnergyProbe:
    """The potential energy per site of generated fields and its gradient,
    from the MD's own force evaluation (mirror_force_mirror: V and dVddi =
    dV/du): one mixed-precision context per pressure, its uniform field set
    per sample.  make_params(L, T, E_z, GPa) as experiment takes it."""

    def __init__(self, make_params, L):
        self.make_params = make_params
        self.L = L
        self.ctx = {}

    def _context(self, gpa):
        import feram_b200 as fb
        if gpa not in self.ctx:
            p = self.make_params(self.L, 300.0, 0.0, gpa)
            c = fb.Context(p, FG_PREC_MIXED)
            c.build_tables()
            self.ctx[gpa] = (c, p)
        return self.ctx[gpa]

    def __call__(self, net, cond):
        """(V/N [batch], dV/du / N [batch][N][3]) of the last forward's fields."""
        V, G = [], []
        for b, c in enumerate(np.asarray(cond)):
            ctx, p = self._context(float(c[4]))
            ctx.set_state(net.field(b, p))
            ctx.set_uniform_E([c[1], c[2], c[3]])
            e = ctx.mirror_force_mirror()
            V.append(potential(e) / p.N)
            G.append(A.physical(ctx.get_state()["dVddi"], p).reshape(-1, 3) / p.N)
        return np.array(V), np.array(G)

    def close(self):
        for c, _ in self.ctx.values():
            c.close()
        self.ctx = {}


def train(net: WarmStartNet, cond, stats, steps=1500, lr=2e-3, seed=0, log_every=0, energies=None, probe=None,
          energy_from=None):
    """Adam on the moment-matching loss, minibatches of net.batch training
    samples (random order, fresh noise seeds).  Weights: 1 / variance of
    each statistic over the training set.  With energies (V/N of each
    training configuration) and an EnergyProbe, the steps from energy_from
    (default: half way) on add w_V (V/N - V_target)^2 per sample (w_V: 1 /
    variance of V/N), whose gradient is the MD force of the generated field:
    the statistics alone leave the fields smoother than thermal ones (their
    potential energy too low).  Returns the loss history (statistics, plus
    the energy term where it is on)."""
    rng = np.random.default_rng(seed)
    w = 1.0 / np.maximum(stats.var(axis=0), 1e-30)
    use_e = energies is not None and probe is not None
    wv = 1.0 / max(float(np.var(energies)), 1e-30) if use_e else 0.0
    e_from = steps // 2 if energy_from is None else energy_from
    hist = []
    for it in range(steps):
        idx = rng.integers(0, len(cond), size=net.batch)
        seeds = rng.integers(1, 2 ** 62, size=net.batch)
        lr_t = lr * (0.1 ** (it / max(steps, 1)))  # exponential decay to lr / 10
        if use_e and it >= e_from:
            net.forward(cond[idx], seeds)
            V, G = probe(net, cond[idx])
            d = V - energies[idx]
            dLdu = (2.0 * wv / net.batch) * d[:, None, None] * G
            loss = net.backward(cond[idx], seeds, stats[idx], w, dLdu) + wv * float(np.mean(d * d))
        else:
            loss = net.backward(cond[idx], seeds, stats[idx], w)
        net.adam(lr_t)
        hist.append(loss)
        if log_every and it % log_every == 0:
            print(f"train step {it}: loss {loss:.4g}", flush=True)
    return np.array(hist)


def equilibration_trace(ctx, n_steps: int, every: int):
    """(|<u>|^2, potential energy) every `every` steps over n_steps, from
    the device reductions of add_to_Average (fg_average_accumulate)."""
    P2, V = [], []
    N = ctx.p.Lx * ctx.p.Ly * ctx.p.Lz
    for _ in range(n_steps // every):
        e = ctx.run_steps(every)
        avg = A.fg_average()
        ctx.average_accumulate(e, avg)
        m = np.array(avg.u[:]) / N
        P2.append(float(m @ m))
        V.append(potential(e))
    return np.array(P2), np.array(V)


def time_to_equilibrium(P2, V, eq, every: int, block: int = 5, k: float = 3.0):
    """Steps until three consecutive blocks (block samples each) of the trace
    lie within k standard deviations (of block means) of the equilibrium
    values eq = (P2 mean, P2 block sd, V mean, V block sd); None if never."""
    nb = len(P2) // block
    bp = P2[:nb * block].reshape(nb, block).mean(axis=1)
    bv = V[:nb * block].reshape(nb, block).mean(axis=1)
    ok = (np.abs(bp - eq[0]) <= k * eq[1] + 1e-12) & (np.abs(bv - eq[2]) <= k * eq[3] + 1e-12)
    for i in range(nb - 2):
        if ok[i] and ok[i + 1] and ok[i + 2]:
            return i * block * every
    return None


def block_stats(P2, V, block: int = 5):
    nb = len(P2) // block
    bp = P2[:nb * block].reshape(nb, block).mean(axis=1)
    bv = V[:nb * block].reshape(nb, block).mean(axis=1)
    return (float(bp.mean()), float(bp.std(ddof=1)), float(bv.mean()), float(bv.std(ddof=1)))


def accept(Pw, Vw, Pe, Ve, k: float = 4.0, block: int = 5) -> bool:
    """The MD as the referee of a warm start: the warm run's block-averaged
    |<u>|^2 and potential energy against the plain run's equilibrium, each
    within k standard errors of their difference (block means of `block`
    samples); a rejected warm start keeps the chained fallback."""
    a, e = block_stats(Pw, Vw, block), block_stats(Pe, Ve, block)
    na, ne = len(Pw) // block, len(Pe) // block
    return bool(abs(a[0] - e[0]) <= k * np.hypot(a[1] / np.sqrt(na), e[1] / np.sqrt(ne)) + 1e-12 and
                abs(a[2] - e[2]) <= k * np.hypot(a[3] / np.sqrt(na), e[3] / np.sqrt(ne)) + 1e-12)


def timed(fn, *a, **k):
    t0 = time.perf_counter()
    r = fn(*a, **k)
    return r, time.perf_counter() - t0


def settle(ctx, T, E, n_vs):
    """n_vs steps of velocity scaling (velocity_scaling.F:9-103: the kinetic
    energy held at the target every step) from a proposed state, then the
    point's Nose-Poincare start (fg_chain_point: force, s = 1, pi = 0, H0).
    A proposal whose potential energy is off relaxes against the rescaled
    momenta in a few hundred steps instead of through the slow thermostat."""
    e = A.fg_energy()
    for _ in range(n_vs):
        ctx.velocity_scaling(e)
    ctx.chain_point(T, E)


def _sweep(net, make_params, L, points, seed, probe, every, accept_after, say, tag, n_vs=0):
    """One pass over held-out points in the given order: for each, the
    fallback (chained from the previous point), the network's warm start and
    a cold start (initialize_dipoR's uni64 field, p = 0), each of the last
    two settled by n_vs velocity-scaling steps (counted in its time), then
    `probe` Nose-Poincare steps each.  The equilibrium every start is judged
    against comes from an independent chain through the same points (another
    uni64 seed), thermalised `probe` steps at each point and then measured
    over `probe` more: not from the fallback's own continuation, which would
    share the fallback's slow fluctuations and favour it."""
    import feram_b200 as fb
    p0 = make_params(L, points[0][0], points[0][1], -5.0)
    rows, t_infer = [], 0.0
    with fb.Context(p0, FG_PREC_MIXED) as cf, fb.Context(p0, FG_PREC_MIXED) as cw, \
            fb.Context(p0, FG_PREC_MIXED) as cc, fb.Context(p0, FG_PREC_MIXED) as ce:
        for c in (cf, cw, cc, ce):
            c.build_tables()
        for c, s1 in ((cf, p0.seed[0]), (ce, p0.seed[0] + 1)):
            pi = A.fg_params.from_buffer_copy(p0)
            pi.seed[0] = s1
            u = A.real_field(pi)
            q = A.real_field(pi)
            assert A.lib().fg_init_dipoR_host(C.byref(pi), A.dptr(u), A.dptr(q)) == 0
            start_point(c, p0, u, q)
            c.run_steps(probe)  # the sweep's first point, thermalised before the held-out ones
        for i, (T, ez) in enumerate(points):
            E = [0.0, 0.0, ez]
            cf.chain_point(T, E)
            Pf, Vf = equilibration_trace(cf, probe, every)
            ce.chain_point(T, E)
            ce.run_steps(probe)
            Pe, Ve = equilibration_trace(ce, probe, every)
            eq = block_stats(Pe, Ve)
            t0 = time.perf_counter()
            net.forward(np.array([[T, 0.0, 0.0, ez, -5.0]] * net.batch), [seed * 1000 + i] * net.batch)
            pw = make_params(L, T, ez, -5.0)
            uw = net.field(0, pw)
            t_infer += time.perf_counter() - t0
            cw.chain_point(T, E)  # the context's temperature and field; its state is replaced
            start_point(cw, cw.p, uw, maxwell_momenta(cw.p, seed + i))
            settle(cw, T, E, n_vs)
            Pw, Vw = equilibration_trace(cw, probe, every)
            cc.chain_point(T, E)
            pc = A.fg_params.from_buffer_copy(cc.p)
            pc.seed[0] = 123456789 + i
            uc = A.real_field(pc)
            assert A.lib().fg_init_dipoR_host(C.byref(pc), A.dptr(uc), None) == 0
            start_point(cc, cc.p, uc, A.real_field(pc))
            settle(cc, T, E, n_vs)
            Pc, Vc = equilibration_trace(cc, probe, every)
            tf = time_to_equilibrium(Pf, Vf, eq, every)
            tw = time_to_equilibrium(Pw, Vw, eq, every)
            tc = time_to_equilibrium(Pc, Vc, eq, every)
            k0 = accept_after // every
            ok = accept(Pw[k0:], Vw[k0:], Pe, Ve)
            val = lambda t, extra=0: extra + (probe if t is None else t)
            Nn = cw.p.N
            rows.append([T, ez, val(tf), val(tw, n_vs), val(tc, n_vs), int(ok), Vf[0] / Nn, Vw[0] / Nn, eq[2] / Nn,
                         float(Pf[0]), float(Pw[0]), eq[0]])
            say(f"  {tag} point {i}: T {T:.1f} K, E_z {ez:+.5f}: tau fallback {val(tf)}, warm {val(tw, n_vs)}, "
                f"cold {val(tc, n_vs)}, {'accepted' if ok else 'rejected'}")
    r = np.array(rows)
    tf, tw, tc, acc = r[:, 2], r[:, 3], r[:, 4], r[:, 5]
    eff = np.where(acc == 1, tw, tw + tf)  # a rejected warm start pays both tries
    return {"points": len(rows), "accepted": int(acc.sum()),
            "tau_fallback_median": float(np.median(tf)), "tau_warm_median": float(np.median(tw)),
            "tau_cold_median": float(np.median(tc)), "tau_fallback_mean": float(tf.mean()),
            "tau_warm_mean": float(tw.mean()), "tau_cold_mean": float(tc.mean()),
            "warm_faster_than_fallback": int(np.sum(tw < tf)), "warm_faster_than_cold": int(np.sum(tw < tc)),
            "thermalisation_steps_fallback": int(tf.sum()), "thermalisation_steps_warm_with_fallback": int(eff.sum()),
            "thermalisation_steps_cold": int(tc.sum()), "inference_seconds": t_infer,
            "rows": [[round(x, 6) for x in row] for row in rows]}


def experiment(make_params, L=32, train_chains=None, train_temps=None, n_held=40, n_shuffled=20, seed=2024,
               n_therm=3000, n_snap=14, train_steps=4000, probe=3000, every=20, accept_after=1000, log=None,
               keep_layers=False, energy_from=3000, n_vs=200):
    """The learned-warm-start protocol on one GPU.

    1. Data: MD cooling chains (train_chains of (E_z, GPa), train_temps
       descending) at L^3, snapshots -> (condition, statistics).
    2. Training: Adam on the moment-matching loss; from step energy_from
       on (None: never) also on the potential energy per site, with the
       MD force as its gradient (EnergyProbe).
    3. Held-out points (T in 100-450 K, E_z in +-0.001 V/A), off the
       training grid: n_held visited as a cooling sweep (T descending) and
       n_shuffled in random order (a scan whose previous point is unrelated).
       Each point runs from the previous point's final state (fg_chain_point,
       the reference's .restart chaining: the fallback), from the network's
       proposal with Maxwell-Boltzmann momenta, and from a cold uni64 start
       (both settled by n_vs velocity-scaling steps, counted in their times);
       an independent chain through the same points gives the point's
       equilibrium (block means and their spread).  Time to equilibrium: three consecutive blocks of the
       trace within 3 sigma of it.  Acceptance, the MD as the referee: the warm
       run's averages over [accept_after, probe) against the equilibrium,
       within 4 sigma of the difference; a rejected point keeps the fallback.
    Returns a dict of the measurements (with keep_layers, "_layers": the
    trained [(w, b)] of the four layers); the "rows" of each pass are (T, E_z,
    tau fallback, tau warm, tau cold, accepted, V/N of the first fallback
    and warm samples, equilibrium V/N, the same three for |<u>|^2)."""
    say = log or (lambda *a: None)
    rng = np.random.default_rng(seed)
    if train_chains is None:
        train_chains = [(ez, gpa) for ez in (-0.001, -0.0005, 0.0, 0.0005, 0.001) for gpa in (-5.0, -3.0)]
    if train_temps is None:
        train_temps = [450.0 - 25.0 * i for i in range(15)]
    out = {"L": L, "train_chains": len(train_chains), "train_temps": [train_temps[0], train_temps[-1], len(train_temps)]}
    (cond, stats, energies), t_data = timed(generate_training_set, lambda T, ez, gpa: make_params(L, T, ez, gpa),
                                  train_chains, train_temps, n_therm=n_therm, n_snap=n_snap)
    out["train_configs"] = len(cond)
    out["data_seconds"] = t_data
    say(f"warm start: {len(cond)} training configurations in {t_data:.1f} s")
    net = WarmStartNet((L, L, L), batch=8, seed=seed)
    try:
        probe_e = EnergyProbe(make_params, L) if energy_from is not None else None
        try:
            hist, t_train = timed(train, net, cond, stats, steps=train_steps, seed=seed, energies=energies,
                                  probe=probe_e, energy_from=energy_from)
        finally:
            if probe_e is not None:
                probe_e.close()
        out["energy_matching_from_step"] = energy_from
        out.update({"train_steps": train_steps, "train_seconds": t_train,
                    "loss_first": float(np.mean(hist[:20])), "loss_last": float(np.mean(hist[-50:]))})
        say(f"warm start: trained {train_steps} steps in {t_train:.1f} s, loss {out['loss_first']:.3g} -> "
            f"{out['loss_last']:.3g}")
        pts = [(float(rng.uniform(100.0, 450.0)), float(rng.uniform(-0.001, 0.001))) for _ in range(n_held + n_shuffled)]
        out["settle_vs_steps"] = n_vs
        out["cooling_sweep"] = _sweep(net, make_params, L, sorted(pts[:n_held], reverse=True), seed, probe, every,
                                      accept_after, say, "sweep", n_vs)
        if n_shuffled > 0:
            out["shuffled"] = _sweep(net, make_params, L, pts[n_held:], seed + 7, probe, every, accept_after, say,
                                     "shuffled", n_vs)
        if keep_layers:
            out["_layers"] = [net.layer(l)[:2] for l in range(4)]
    finally:
        net.close()
    return out
