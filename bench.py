#!/usr/bin/env python
"""MD site-steps/s of feram's Nose-Poincare step at 128^3 on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: bulk BaTiO3 effective Hamiltonian (the Zhong-Vanderbilt-Rabe
parameter set of the reference's BaTiO3 cooling example), 128^3 supercell,
300 K, dt = 2 fs, E_z = 100 kV/cm, Nose-Poincare (method 'md').  The initial
dipoles are uni64-seeded Gaussians (sigma 0.03 A); one step = one full
nose_poincare call (kick, thermostat, drift, force, kick).  The timed steps
run as CUDA graphs on the library's own stream and are timed with CUDA
events recorded on that stream; the working set (fields, spectra and tables,
~0.3 GB in the mixed path) exceeds the 126 MB L2, so no flush is needed.

Under torchrun each rank runs an independent replica on its own GPU (the
reference's task-farm parallelism, replicas only); value is the whole-job
rate and the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MD site-steps/s at 128^3: mixed vs FP64 GPU (force err<=1e-6); % HBM peak"
UNIT = "site-steps/s"
L_DEFAULT = 128
# fg_nose_poincare calls in the end-to-end measurement, independent of --steps:
# the run length of the 128^3 workload (1e4 steps), over which the one upload
# and one download of the whole state are spread
E2E_STEPS = 10000

# BaTiO3, Zhong-Vanderbilt-Rabe effective-Hamiltonian parameters as used by
# the reference's BaTiO3 cooling sweep and 64^3 benchmark input decks (eV,
# Angstrom, ps).  The Nose-Poincare mass grows with the supercell: the 64^3
# benchmark deck uses Q = 1.0, so Q = 1.0 * N / 64^3 here (8.0 at 128^3),
# which keeps CB dt / Q of nose-poincare.F:36 far below 1.
ZVR = dict(GPa=-5.0, mass_amu=39.0, Q_Nose_64=1.0, a0=3.94, dt=0.002,
           P_kappa2=5.502, P_alpha=110.4, P_gamma=-163.1,
           j=(-2.648, 3.894, 0.898, -0.789, 0.562, 0.358, 0.179),
           B11=126.0, B12=44.9, B44=50.3, B1xx=-211.0, B1yy=-19.3, B4yz=-7.75,
           Z_star=9.956, epsilon_inf=5.24)


def _param_lib(impl):
    """(defaults, make) of the arm: the product's host code for ours, the
    oracle's own restatement of read_Param/make_Param for the reference arm,
    so that the reference process never loads the product library."""
    from feram_b200 import _capi as A
    if impl == "ours":
        import feram_b200 as fb
        return fb.default_params, fb.make_param
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    L = oracle_lib.load()

    def defaults():
        p = A.fg_params()
        L.oracle_default_param(C.byref(p))
        return p

    def make(p):
        assert L.oracle_make_param(C.byref(p)) == 0
        return p
    return defaults, make


def make_params(L, kelvin=300.0, Ez=0.001, seed=(123456789, 987654321), impl="ours"):
    defaults, make = _param_lib(impl)
    p = defaults()
    z = ZVR
    p.method = 0
    p.GPa[0] = p.GPa[1] = p.GPa[2] = z["GPa"]
    p.kelvin = kelvin
    for s in range(3):
        p.mass_dipo[s] = z["mass_amu"] / 9648.53377163899
        p.P_kappa2[s], p.P_alpha[s], p.P_gamma[s] = z["P_kappa2"], z["P_alpha"], z["P_gamma"]
        p.Z_star[s] = z["Z_star"]
        p.init_dipo_dev[s] = 0.03
        p.init_dipo_avg[s] = 0.0
    p.Q_Nose = z["Q_Nose_64"] * L ** 3 / 64 ** 3
    p.a0, p.dt = z["a0"], z["dt"]
    p.Lx = p.Ly = p.Lz = L
    for i, v in enumerate(z["j"]):
        p.j[i] = v
    p.B11, p.B12, p.B44, p.B1xx, p.B1yy, p.B4yz = (z[k] for k in ("B11", "B12", "B44", "B1xx", "B1yy", "B4yz"))
    p.epsilon_inf = z["epsilon_inf"]
    p.external_E_field[2] = Ez
    p.E_field_always_zero = 0 if Ez != 0.0 else 1
    p.seed[0], p.seed[1] = seed
    return make(p)


def initial_state(p, impl="ours"):
    """initialize_dipoR's seeded u and p = 0 (product host code, or the
    oracle's restatement for the reference arm)."""
    from feram_b200 import _capi as A
    u = A.real_field(p)
    q = A.real_field(p)
    if impl == "ours":
        assert A.lib().fg_init_dipoR_host(C.byref(p), A.dptr(u), A.dptr(q)) == 0
    else:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib
        assert oracle_lib.load().oracle_init_dipoR(C.byref(p), A.dptr(u), A.dptr(q)) == 0
    return u, q


def loaded_repo_libs():
    """Shared objects of this repository mapped into the process."""
    libs = set()
    try:
        for line in open("/proc/self/maps"):
            path = line.split()[-1] if len(line.split()) >= 6 else ""
            if path.endswith(".so") and os.path.abspath(path).startswith(ROOT):
                libs.add(os.path.relpath(path, ROOT))
    except OSError:
        return None
    return sorted(libs)


def rank_layout():
    """(world size, rank, local rank) from the launcher's environment
    (torchrun sets them; a plain run is rank 0 of 1)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(rank):
    """uni64 seeds of the replica on `rank`: an independent replica per rank,
    as the reference's feram_mpi task farm runs one input per rank."""
    return (123456789 + rank, 987654321)


def reduce_max(v, world, dist=None, device="cuda"):
    """The maximum of v over the ranks (all_reduce MAX of one FP64 value)."""
    if world == 1:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job(sites_per_rank, steps, ms_max, world):
    """Site-steps per second of the whole job: every rank's sites and steps
    over the slowest rank's time (weak scaling: work per rank fixed)."""
    return sites_per_rank * steps * world / (ms_max * 1e-3)


def bench_config(L, sites, world):
    """The workload description both arms print."""
    return {"workload": f"{L}^3 bulk BaTiO3 Nose-Poincare MD, 300 K, dt 2 fs, E_z 100 kV/cm",
            "sites": sites, "precision": "mixed", "parallelism": f"replicas x{world}",
            "l2": "working set > 126 MB L2, no flush"}


def fp32_config(u):
    """u rounded to FP32: the configuration the mixed path holds."""
    return u.astype(np.float32).astype(np.float64)


ENERGY_TERMS = ("short_range", "long_range", "dipole_E_field", "unharmonic", "homo_strain", "homo_coupling",
                "inho_strain", "inho_coupling")


def force_errors_16(ctxm, ctx64, p, sigma=0.1):
    """Mixed against FP64 force and energies on 16 fixed configurations,
    u ~ N(0, sigma) per component from uni64 seeds (s, 987654321), s = 1..16,
    rounded to FP32 (the state the mixed path holds) and given identically to
    both paths; the FP64 path matches the oracle to 1e-12.  Force errors:
    max |dF| / rms |F| over sites (worst site against the typical force), rms
    |dF| / rms |F| (relative L2 norm) and max |dF| / max |F| (relative max
    norm); energy error per term over the sum of the terms' magnitudes.
    state_rounding: the same worst-site measure between the FP64 forces of
    the unrounded and the FP32-rounded configuration, i.e. what holding u in
    FP32 at all moves the force by (a property of FP32 state, not of the
    mixed arithmetic)."""
    from feram_b200 import _capi as A
    worst = {"max": 0.0, "rms": 0.0, "maxnorm": 0.0, "energy": 0.0, "state": 0.0}
    for s in range(1, 17):
        q = A.fg_params.from_buffer_copy(p)
        q.seed[0], q.seed[1] = s, 987654321
        for a in range(3):
            q.init_dipo_avg[a], q.init_dipo_dev[a], q.k_stripe[a] = 0.0, sigma, 0.0
        u64 = A.real_field(p)
        assert A.lib().fg_init_dipoR_host(C.byref(q), A.dptr(u64), None) == 0
        u = fp32_config(u64)
        es, fs = [], []
        for ctx in (ctx64, ctxm):
            ctx.set_state(u)
            es.append(ctx.mirror_force_mirror())
            fs.append(A.physical(ctx.get_state()["dVddi"], p).copy())
        ctx64.set_state(u64)
        ctx64.mirror_force_mirror()
        f64u = A.physical(ctx64.get_state()["dVddi"], p)
        d = np.sqrt(np.sum((fs[1] - fs[0]) ** 2, axis=-1))
        rms = float(np.sqrt(np.mean(np.sum(fs[0] ** 2, axis=-1))))
        scale = sum(abs(getattr(es[0], t)) for t in ENERGY_TERMS)
        worst["max"] = max(worst["max"], float(d.max()) / rms)
        worst["maxnorm"] = max(worst["maxnorm"], float(d.max()) / float(np.sqrt(np.sum(fs[0] ** 2, axis=-1)).max()))
        worst["rms"] = max(worst["rms"], float(np.sqrt(np.mean(d ** 2))) / rms)
        worst["energy"] = max(worst["energy"],
                              max(abs(getattr(es[1], t) - getattr(es[0], t)) for t in ENERGY_TERMS) / scale)
        worst["state"] = max(worst["state"], float(np.sqrt(np.sum((f64u - fs[0]) ** 2, axis=-1)).max()) / rms)
    return {"configs": 16, "sigma": sigma, "seeds": "uni64 (1..16, 987654321), rounded to FP32",
            "force_rms": worst["rms"], "force_maxnorm": worst["maxnorm"], "force_max_site_over_rms": worst["max"],
            "energy_max": worst["energy"], "state_rounding_max_site_over_rms": worst["state"]}


def prepare(ctx, p, u, q):
    """initialize_dipoR's tail and molecular-dynamics.F:209-212 (H0)."""
    ctx.set_state(u, q, 1.0, 0.0, 0.0)
    ctx.set_uniform_E([p.external_E_field[0], p.external_E_field[1], p.external_E_field[2]])
    e = ctx.mirror_force_mirror()
    e.dipo_kinetic = ctx.kinetic_energy_dipo()
    ctx.nose_poincare_hamiltonian(e)
    H0 = e.H_Nose_Poincare
    ctx.set_thermostat(1.0, 0.0, H0)
    ctx.nose_poincare_hamiltonian(e)
    return H0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def kernel_bytes(p, esz):
    """Compulsory DRAM bytes per launch of each kernel of one step (inputs
    read once + outputs written once), esz = bytes per real."""
    N = p.Lx * p.Ly * p.Lz
    nk = (p.Lx // 2 + 1) * p.Ly * p.Lz  # half-spectrum points per component
    c = 2 * esz
    return {
        "k_kick_drift(35a,35c)": 15 * N * esz,
        "k_xy_fwd": 3 * N * esz + 9 * nk * c,
        "k_z_kspace": 18 * nk * c + 6 * nk * esz,
        "k_xy_inv+homo_strain": 9 * nk * c + 9 * N * esz,
        "k_assemble+kick(35e,35f)+np_tail": 21 * N * esz,  # R rw9 u3 p3, W F3 p3
    }


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0}, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes per kernel from the committed ncu summary, if any."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic_128.json")))
    except (OSError, ValueError):
        return {}


def batched_sweep(n_rep=96, steps=200):
    """The batched cooling sweep: n_rep independent replicas of uneven sizes
    (16^3 .. 64^3) on a 450 -> 100 K grid in 5 K steps, mixed precision,
    stepped as one graph (fg_batch_step) and, for comparison, one replica
    after another (fg_run_steps).  Wall-clock seconds around synchronous
    calls; site-steps/s summed over replicas."""
    import feram_b200 as fb
    from feram_b200 import _capi as A
    sizes = [16, 24, 32, 48, 64]
    ps = [make_params(sizes[i % len(sizes)], kelvin=450.0 - 5.0 * (i % 71), Ez=0.0,
                      seed=(123456789 + i, 987654321)) for i in range(n_rep)]
    sites = sum(p.N for p in ps)
    with fb.Batch(ps, A.FG_PREC_MIXED) as b:
        for r, p in zip(b.replicas, ps):
            u, q = initial_state(p)
            r.build_tables()
            prepare(r, p, u, q)
        # one graph branch per replica, then replicas of one size grouped
        # into one launch per kernel (fg_batch_step's default)
        b.set_grouping(False)
        b.step(3)  # warm-up: graph capture and first launches
        t0 = time.perf_counter()
        b.step(steps)
        t_branch = time.perf_counter() - t0
        b.set_grouping(True)
        b.step(3)
        t0 = time.perf_counter()
        b.step(steps)
        t_batch = time.perf_counter() - t0
        groups = b.groups
        # the same grouped graph without branch launch priorities
        b.set_priorities(False)
        b.step(3)
        t0 = time.perf_counter()
        b.step(steps)
        t_noprio = time.perf_counter() - t0
        b.set_priorities(True)
        # the same replicas, one after another (warm-up captures both the
        # eight-step and the one-step graph of fg_run_steps)
        for r in b.replicas:
            r.run_steps(11)
        t0 = time.perf_counter()
        for r in b.replicas:
            r.run_steps(steps)
        t_seq = time.perf_counter() - t0
    return {"replicas": n_rep, "sizes": sizes, "kelvin_grid": [450.0, 100.0, -5.0], "sites": sites, "steps": steps, "precision": "mixed",
            "value": sites * steps / t_batch, "unit": UNIT, "graph_branches": groups,
            "branch_per_replica_value": sites * steps / t_branch,
            "no_branch_priority_value": sites * steps / t_noprio,
            "sequential_value": sites * steps / t_seq, "speedup": t_seq / t_batch,
            "timing": "wall clock around synchronous calls"}


def _block_mean(x, nb=10):
    """Mean and its standard error from nb block means."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x) // nb * nb
    m = x[:n].reshape(nb, -1).mean(axis=1)
    return float(m.mean()), float(m.std(ddof=1) / np.sqrt(nb))


def _point_obs(rows, N):
    """Per-site observables of a point's sample rows: V/N, KE/N, |u_bar|
    (u_bar = sum u / N, the order parameter) and |u_bar|^2."""
    ub = rows[:, 0:3] / N
    a = np.sqrt((ub ** 2).sum(axis=1))
    return {"V": rows[:, 6] / N, "KE": rows[:, 7] / N, "|u|": a, "u2": a * a}


def _ensemble_z(means_a, means_b):
    """z of the difference of two ensemble means (independent replicas)."""
    a, b = np.asarray(means_a), np.asarray(means_b)
    se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
    return float((a.mean() - b.mean()) / max(se, 1e-300)), float(a.mean()), float(b.mean()), float(se)


def sweep_replicas(n_rep):
    """The 96 replicas of the batched sweep: supercell 16^3..64^3 by i mod 5,
    uni64 seeds (123456789 + i, 987654321)."""
    sizes = [16, 24, 32, 48, 64]
    Ls = [sizes[i % len(sizes)] for i in range(n_rep)]
    seeds = [(123456789 + i, 987654321) for i in range(n_rep)]
    return sizes, Ls, seeds


def chained_sweep(n_rep=96, n_points=4, n_therm=1000, n_avg=1000, every=10, log=None):
    """The batched cooling sweep as the reference runs a sweep: every replica
    cools from 450 K in 5 K steps, each point n_therm + n_avg steps started
    from the previous point's final state (cooling.sh:64-69, fg_chain_point
    on the device), mixed precision.

    plain: one replica after another (fg_run_point), default plans.
    batched: all replicas at once, one fg_batch_run_point per temperature
      (grouped launches, plans from fg_batch_tune).
    Agreement: per supercell size and point, the ensemble mean over the
    replicas of that size (independent seeds) of V/N, KE/N, |u_bar| and
    |u_bar|^2, each replica's value its mean over the n_avg steps; z = the
    difference over the ensembles' combined standard error.  Wall clock
    around synchronous calls; set-up (tables, initial state) outside."""
    import feram_b200 as fb
    from feram_b200 import _capi as A
    say = log or (lambda *a: None)
    sizes, Ls, seeds = sweep_replicas(n_rep)
    Ts = [450.0 - 5.0 * k for k in range(n_points)]
    ps = [make_params(Ls[i], kelvin=Ts[0], Ez=0.0, seed=seeds[i]) for i in range(n_rep)]
    sites = sum(p.N for p in ps)
    out = {"replicas": n_rep, "sizes": sizes, "kelvin": Ts, "points": n_points, "sites": sites,
           "n_therm": n_therm, "n_avg": n_avg, "sample_every": every, "precision": "mixed", "unit": UNIT,
           "site_steps": sites * n_points * (n_therm + n_avg),
           "timing": "wall clock around synchronous calls; set-up (tables, initial state) outside"}
    plain = [[None] * n_points for _ in range(n_rep)]
    t_plain = 0.0
    for i in range(n_rep):
        with fb.Context(ps[i], A.FG_PREC_MIXED) as ctx:
            ctx.build_tables()
            u, q = initial_state(ps[i])
            prepare(ctx, ps[i], u, q)
            t0 = time.perf_counter()
            for k in range(n_points):
                ctx.run_point(Ts[k], n_therm, n_avg, every)
                plain[i][k] = ctx.samples()
            t_plain += time.perf_counter() - t0
    say(f"chained sweep: plain sequential {t_plain:.1f} s")
    batched = [[None] * n_points for _ in range(n_rep)]
    with fb.Batch(ps, A.FG_PREC_MIXED) as b:
        for i, r in enumerate(b.replicas):
            r.build_tables()
            u, q = initial_state(ps[i])
            prepare(r, ps[i], u, q)
        t0 = time.perf_counter()
        tb = b.tune(steps=8)
        t_tune = time.perf_counter() - t0
        plans = sorted({(ps[i].Lx,) + b.replicas[i].plan[:2] for i in range(n_rep)})
        t0 = time.perf_counter()
        for k in range(n_points):
            b.run_point([Ts[k]] * n_rep, n_therm, n_avg, every)
            for i, rows in enumerate(b.samples()):
                batched[i][k] = rows
        t_batch = time.perf_counter() - t0
        groups = b.groups
    say(f"chained sweep: batched {t_batch:.1f} s")
    zs, table = [], []
    for L in sizes:
        idx = [i for i in range(n_rep) if Ls[i] == L]
        for k in range(n_points):
            for obs in ("V", "KE", "|u|", "u2"):
                ma = [_point_obs(batched[i][k], ps[i].N)[obs].mean() for i in idx]
                mb = [_point_obs(plain[i][k], ps[i].N)[obs].mean() for i in idx]
                z, a_, b_, se = _ensemble_z(ma, mb)
                zs.append(z)
                table.append([L, Ts[k], obs, round(z, 3), a_, b_, se])
    zs = np.abs(np.array(zs))
    out.update({"plain_seconds": t_plain, "plain_value": out["site_steps"] / t_plain,
                "batched_seconds": t_batch, "batched_value": out["site_steps"] / t_batch,
                "speedup": t_plain / t_batch, "tune_seconds": t_tune, "tune_ms_per_batch_step": list(tb),
                "plans": plans, "graph_branches": groups,
                "agreement": {"comparisons": int(len(zs)), "within_3sigma": int(np.sum(zs <= 3.0)),
                              "max_abs_z": float(zs.max()), "chi2_per_comparison": float(np.mean(zs ** 2)),
                              "rows": table if n_points <= 8 else sorted(table, key=lambda r: -abs(r[3]))[:40]}})
    return out


def parallel_points(n_rep=96, n_therm=1000, n_avg=1000, every=10, warm_layers=None, n_vs=200, log=None):
    """The points of the sweep run at once instead of one after another: n_rep
    points (supercell by i mod 5, T = 450 - 5 (i mod 71) K), each started
    from initialize_dipoR's state (cold) or, with warm_layers, from the
    warm-start network's proposal, settled by n_vs velocity-scaling steps
    (as warm_start.settle; timed with the run), then n_therm + n_avg steps in
    one fg_batch_run_point; against the chained sequential sweep through the same
    points (per supercell, descending T, fg_run_point).  Agreement per point:
    V/N, KE/N, |u_bar|, |u_bar|^2 over the n_avg steps (10 block means),
    z = difference / combined standard error."""
    import feram_b200 as fb
    from feram_b200 import _capi as A
    from feram_b200 import warm_start as W
    say = log or (lambda *a: None)
    sizes, Ls, seeds = sweep_replicas(n_rep)
    Ts = [450.0 - 5.0 * (i % 71) for i in range(n_rep)]
    ps = [make_params(Ls[i], kelvin=Ts[i], Ez=0.0, seed=seeds[i]) for i in range(n_rep)]
    sites = sum(p.N for p in ps)
    out = {"replicas": n_rep, "sizes": sizes, "kelvin": [450.0, 100.0, -5.0], "sites": sites, "n_therm": n_therm,
           "n_avg": n_avg, "sample_every": every, "precision": "mixed", "unit": UNIT,
           "timing": "wall clock around synchronous calls; set-up (tables, initial state) outside"}
    plain = {}
    t_plain = 0.0
    for L in sizes:
        idx = sorted((i for i in range(n_rep) if Ls[i] == L), key=lambda i: -Ts[i])
        p0 = make_params(L, kelvin=Ts[idx[0]], Ez=0.0, seed=seeds[idx[0]])
        with fb.Context(p0, A.FG_PREC_MIXED) as ctx:
            ctx.build_tables()
            u, q = initial_state(p0)
            prepare(ctx, p0, u, q)
            t0 = time.perf_counter()
            for i in idx:
                ctx.run_point(Ts[i], n_therm, n_avg, every)
                plain[i] = ctx.samples()
            t_plain += time.perf_counter() - t0
    out["plain_seconds"] = t_plain
    say(f"parallel points: chained sequential {t_plain:.1f} s")

    def batched_arm(starts, tag):
        with fb.Batch(ps, A.FG_PREC_MIXED) as b:
            for i, r in enumerate(b.replicas):
                r.build_tables()
                u, q = starts(i)
                prepare(r, ps[i], u, q)
            b.tune(steps=8)
            t0 = time.perf_counter()
            e = fb.fg_energy()
            for r in b.replicas:
                for _ in range(n_vs):
                    r.velocity_scaling(e)
            b.run_point(Ts, n_therm, n_avg, every)
            t_run = time.perf_counter() - t0
            rows = b.samples()
        zs = {k: [] for k in ("V", "KE", "|u|", "u2")}
        worst = []
        for i in range(n_rep):
            oa, ob = _point_obs(rows[i], ps[i].N), _point_obs(plain[i], ps[i].N)
            for k in zs:
                ma, ea = _block_mean(oa[k])
                mb, eb = _block_mean(ob[k])
                z = (ma - mb) / max(np.hypot(ea, eb), 1e-300)
                zs[k].append(z)
                if abs(z) > 3.0:
                    worst.append([Ls[i], Ts[i], k, round(float(z), 2), ma, mb])
        agree = {k: {"within_3sigma": int(np.sum(np.abs(v) <= 3.0)), "max_abs_z": float(np.max(np.abs(v)))}
                 for k, v in zs.items()}
        say(f"parallel points: batched ({tag}) {t_run:.1f} s")
        worst.sort(key=lambda w: -abs(w[3]))
        return {"seconds": t_run, "settle_vs_steps": n_vs, "speedup_vs_chained_sequential": t_plain / t_run,
                "agreement": agree,
                "outside_3sigma": worst[:12]}

    out["cold"] = batched_arm(lambda i: initial_state(ps[i]), "cold")
    if warm_layers is not None:
        fields = {}
        t0 = time.perf_counter()
        for L in sizes:
            idx = [i for i in range(n_rep) if Ls[i] == L]
            with W.WarmStartNet((L, L, L), batch=len(idx), seed=7) as net:
                for l, (w, bb) in enumerate(warm_layers):
                    net.set_layer(l, w, bb)
                cond = np.array([[Ts[i], 0.0, 0.0, 0.0, ps[i].GPa[0]] for i in idx])
                net.forward(cond, [1000 + i for i in idx])
                for k, i in enumerate(idx):
                    fields[i] = (net.field(k, ps[i]), W.maxwell_momenta(ps[i], 2000 + i))
        out["warm"] = batched_arm(lambda i: fields[i], "warm")
        out["warm"]["inference_seconds"] = time.perf_counter() - t0
    return out


def fft_vs_cufft(L=128, reps=20):
    """The device FFT stage (3-component r2c and c2r: k_xy_fwd + z pass, z
    pass + k_xy_inv; fg_time_fft) against cuFFT on the same GPU, planned as
    the reference's cufft_check.F:180-207 plans it (D2Z / Z2D, howmany 3,
    interleaved components, padded embeds) and, as cuFFT's own best case,
    three contiguous unpadded fields.  CUDA events; ms per transform."""
    import torch
    import feram_b200 as fb
    from feram_b200 import _capi as A
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import cufft_lib
    p = make_params(L, Ez=0.0)
    out = {"L": L, "components": 3, "reps": reps}
    for prec, name, fp64 in ((A.FG_PREC_MIXED, "fp32", False), (A.FG_PREC_FP64, "fp64", True)):
        with fb.Context(p, prec) as ctx:
            ms = ctx.time_fft(reps)
        dt, ct = (torch.float64, torch.complex128) if fp64 else (torch.float32, torch.complex64)
        res = {"ours_r2c_ms": ms[0], "ours_c2r_ms": ms[1]}
        for layout in ("reference", "contiguous"):
            if layout == "reference":
                x = torch.zeros(A.real_field(p).shape, dtype=dt, device="cuda")
                X = torch.zeros(A.complex_field(p).shape, dtype=ct, device="cuda")
            else:
                x = torch.zeros((3, L, L, L), dtype=dt, device="cuda")
                X = torch.zeros((3, L, L, L // 2 + 1), dtype=ct, device="cuda")
            x.normal_()
            plan = cufft_lib.PlanMany(L, L, L, 1, 3, fp64, layout)
            try:
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                tf = tb = 0.0
                for r in range(reps + 1):
                    ev[0].record()
                    plan.forward(x.data_ptr(), X.data_ptr())
                    ev[1].record()
                    plan.backward(X.data_ptr(), x.data_ptr())
                    ev[2].record()
                    torch.cuda.synchronize()
                    if r > 0:
                        tf += ev[0].elapsed_time(ev[1])
                        tb += ev[1].elapsed_time(ev[2])
            finally:
                plan.close()
            res[f"cufft_{layout}_r2c_ms"] = tf / reps
            res[f"cufft_{layout}_c2r_ms"] = tb / reps
        res["cufft_reference_over_ours"] = (res["cufft_reference_r2c_ms"] + res["cufft_reference_c2r_ms"]) / (ms[0] + ms[1])
        res["cufft_contiguous_over_ours"] = (res["cufft_contiguous_r2c_ms"] + res["cufft_contiguous_c2r_ms"]) / (ms[0] + ms[1])
        out[name] = res
    return out


def epit_hysteresis(n_rep=16, L=64, steps=400, period=20000):
    """The batched thin-film hysteresis workload: n_rep epitaxial films of
    L x L x L sites (L/2 layers and their mirror image in z), misfit strain
    on a grid from -2% to +2%, a triangular_cos E_z wave of amplitude
    0.002 V/A (200 kV/cm) and period `period` steps evaluated on the device
    every step (fg_set_wave), 300 K, Nose-Poincare, mixed precision, all
    replicas as one batch graph.  `steps` timed steps (of the 2e4 a full loop
    takes); wall clock around the synchronous fg_batch_step."""
    import feram_b200 as fb
    from feram_b200 import _capi as A
    ps = []
    for i in range(n_rep):
        p = make_params(L, kelvin=300.0, Ez=0.002)
        p.bulk_or_film = A.FG_EPIT
        p.epi_strain = -0.02 + 0.04 * i / max(n_rep - 1, 1)
        p.E_wave_type = A.FG_WAVE_TRIANGULAR_COS
        p.n_E_wave_period = period
        p.n_thermalize = 0
        p.seed[0] = 123456789 + i
        ps.append(fb.make_param(p))
    sites = sum(p.N for p in ps)
    with fb.Batch(ps, A.FG_PREC_MIXED) as b:
        for r, p in zip(b.replicas, ps):
            u, q = initial_state(p)
            r.build_tables()
            prepare(r, p, u, q)
            r.set_wave(True, 0)
        b.step(5)
        t0 = time.perf_counter()
        es = b.step(steps)
        t = time.perf_counter() - t0
    return {"replicas": n_rep, "L": [L, L, L], "layers": L // 2, "epi_strain": [-0.02, 0.02],
            "E_wave": "triangular_cos, 0.002 V/A, period %d steps, on the device" % period, "kelvin": 300.0,
            "sites": sites, "steps": steps, "value": sites * steps / t, "unit": UNIT,
            "ms_per_batch_step": 1000.0 * t / steps, "timing": "wall clock around synchronous fg_batch_step",
            "finite": bool(all(np.isfinite(e.total) for e in es))}


def warm_start_leg(L=32, log=None):
    """The learned warm start (32^3): MD-generated training set, training on
    the tensor cores, 40 held-out (T, E) points against the chained
    fallback (feram_b200.warm_start.experiment)."""
    from feram_b200 import warm_start as W

    def mp(Lw, T, ez, gpa):
        import feram_b200 as fb
        p = make_params(Lw, kelvin=T, Ez=ez)
        p.GPa[0] = p.GPa[1] = p.GPa[2] = gpa
        p.E_field_always_zero = 0
        p.N = 0
        return fb.make_param(p)
    return W.experiment(mp, L=L, log=log, keep_layers=True)


def cpu_baseline(p, budget_s=20.0):
    """The oracle (FP64 C++/OpenMP restatement of the reference's CPU path)
    on this host's cores: one NP step after setup, then as many more as fit
    in the budget.  Bounded sample of the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    threads = os.cpu_count() or 1
    oracle_lib.load().oracle_set_threads(threads)
    u, q = initial_state(p)
    o = oracle_lib.Oracle(p)
    o.set_state(u, q)
    o.set_uniform_E([p.external_E_field[0], p.external_E_field[1], p.external_E_field[2]])
    e = o.force()
    e.dipo_kinetic = o.kinetic_energy_dipo()
    o.md(1, 0, 1, e)  # H0
    t0 = time.perf_counter()
    o.nose_poincare(e)
    t1 = time.perf_counter()
    n = 1 + max(0, int((budget_s - (t1 - t0)) / max(t1 - t0, 1e-6)))
    n = min(n, 50)
    for _ in range(n - 1):
        o.nose_poincare(e)
    t2 = time.perf_counter()
    o.close()
    return {"value": p.N * n / (t2 - t0), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} Nose-Poincare steps at {p.Lx}^3 after table setup (oracle/, FP64, OpenMP)"}


def run_reference(args):
    """--impl reference: the reference's CPU path (its C++ restatement, since
    the Fortran/FFTW binary cannot be built here) on all host cores.  Inputs
    come from the oracle's own read_Param/make_Param/initialize_dipoR, so
    nothing of the product is loaded in this process."""
    world, rank, _ = rank_layout()
    if rank != 0:
        return 0
    L = args.size
    p = make_params(L, impl="reference")
    budget = 120.0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    threads = os.cpu_count() or 1
    oracle_lib.load().oracle_set_threads(threads)
    u, q = initial_state(p, impl="reference")
    o = oracle_lib.Oracle(p)
    o.set_state(u, q)
    o.set_uniform_E([0.0, 0.0, p.external_E_field[2]])
    e = o.force()
    e.dipo_kinetic = o.kinetic_energy_dipo()
    o.md(1, 0, 1, e)
    for _ in range(min(args.warmup, 1)):
        o.nose_poincare(e)
    t0 = time.perf_counter()
    o.nose_poincare(e)
    t1 = time.perf_counter()
    n = max(1, min(args.steps, int(budget / max(t1 - t0, 1e-6))))
    for _ in range(n - 1):
        o.nose_poincare(e)
    t2 = time.perf_counter()
    value = p.N * n / (t2 - t0)
    sample = f"{n} of {args.steps} requested Nose-Poincare steps at {L}^3 (FP64 C++/OpenMP restatement)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": n, "warmup": min(args.warmup, 1), "ms_per_step": 1000.0 * (t2 - t0) / n,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: uni64-seeded dipoles, BaTiO3 ZVR parameters",
        "config": bench_config(L, p.N, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "repo_libs_loaded": loaded_repo_libs(),
    }), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=L_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 96-replica batched sweep measurement")
    ap.add_argument("--sweep-points", type=int, default=4,
                    help="temperatures of the chained batched sweep from 450 K down in 5 K steps (71: to 100 K)")
    ap.add_argument("--sweep-only", action="store_true",
                    help="run the chained batched sweep alone and print its JSON object")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the FFT-vs-cuFFT, thin-film hysteresis and warm-start legs")
    ap.add_argument("--mixed-only", action="store_true",
                    help="skip the FP64 context, the force-error check and e2e (small device footprint, for profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.sweep_only:
        out = chained_sweep(n_points=args.sweep_points, log=lambda m: print(m, file=sys.stderr, flush=True))
        print(json.dumps({"cooling_sweep": out}), flush=True)
        return 0

    import torch
    import torch.distributed as dist
    import feram_b200 as fb
    from feram_b200 import _capi as A

    world, rank, local = rank_layout()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        return reduce_max(v, world, dist, "cuda")

    L = args.size
    p = make_params(L, seed=replica_seed(rank))
    u, q = initial_state(p)

    ctxm = fb.Context(p, A.FG_PREC_MIXED)
    ctxm.build_tables()
    H0 = prepare(ctxm, p, u, q)
    ctx64, ferr, ferr16 = None, None, None
    if not args.mixed_only:
        # force error of the mixed path against the FP64 path on the same state
        ctx64 = fb.Context(p, A.FG_PREC_FP64)
        ctx64.build_tables()
        prepare(ctx64, p, fp32_config(u), q)
        f64 = ctx64.get_state()["dVddi"]
        fmx = ctxm.get_state()["dVddi"]
        d = A.physical(fmx, p) - A.physical(f64, p)
        rms = float(np.sqrt(np.mean(np.sum(A.physical(f64, p) ** 2, axis=-1))))
        dn = np.sqrt(np.sum(d ** 2, axis=-1))
        fmaxn = float(np.sqrt(np.sum(A.physical(f64, p) ** 2, axis=-1)).max())
        ferr = {"rms": float(np.sqrt(np.mean(dn ** 2)) / rms), "maxnorm": float(dn.max()) / fmaxn,
                "max_site_over_rms": float(dn.max() / rms)}
        ferr16 = force_errors_16(ctxm, ctx64, p)
        prepare(ctxm, p, u, q)
        prepare(ctx64, p, u, q)

    def timed(ctx, steps, warmup, sample_clocks):
        ms = C.c_double()
        ctx._check(A.lib().fg_time_steps(ctx._h, warmup, C.byref(ms)))
        barrier()
        sampler = ClockSampler(torch.cuda.current_device()) if sample_clocks else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        barrier()
        ctx._check(A.lib().fg_time_steps(ctx._h, steps, C.byref(ms)))
        barrier()
        clocks = sampler.stop() if sampler else None
        return max_over_ranks(ms.value), clocks

    ms_mixed, clocks = timed(ctxm, args.steps, args.warmup, True)
    value = whole_job(p.N, args.steps, ms_mixed, world)
    steps64 = max(args.steps // 2, 10)
    ms_fp64, value64 = None, None
    if ctx64 is not None:
        ms_fp64, _ = timed(ctx64, steps64, args.warmup, False)
        value64 = whole_job(p.N, steps64, ms_fp64, world)

    # per-kernel times of one step (events between kernels, same stream)
    nprof = A.FG_NPROF
    prof = (C.c_double * nprof)()
    ctxm._check(A.lib().fg_profile_step(ctxm._h, 20, prof))
    names = [A.lib().fg_profile_name(i).decode() for i in range(nprof)]
    kb = kernel_bytes(p, 4)
    pk, pk_kind = peaks()
    hbm = float(pk.get("hbm_gbs", 6650.0))
    per_kernel = {}
    for n, t in zip(names, prof):
        ent = {"ms": t}
        if n in kb and t > 0:
            ent["GBps"] = kb[n] / (t * 1e-3) / 1e9
            ent["frac"] = ent["GBps"] / hbm
        per_kernel[n] = ent
    dom = max((n for n in names if n in kb), key=lambda n: per_kernel[n]["ms"])
    traffic = ncu_traffic().get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": per_kernel[dom]["GBps"], "peak": hbm, "unit": "GB/s",
                "frac": per_kernel[dom]["frac"], "peak_kind": pk_kind,
                "algorithmic_bytes": kb[dom], "traffic": traffic}
    ms_step = ms_mixed / args.steps
    step_roofline = {"algorithmic_bytes_per_site_step": 264, "achieved_GBps": 264 * p.N / (ms_step * 1e-3) / 1e9,
                     "frac": 264 * p.N / (ms_step * 1e-3) / 1e9 / hbm,
                     "fp64_frac": (528 * p.N / (ms_fp64 / steps64 * 1e-3) / 1e9 / hbm) if ms_fp64 else None}

    e2e = None
    if not args.mixed_only:
        # e2e through the public C-ABI with host buffers: upload the state from
        # pinned memory, K reference-style per-step calls (field H2D, energies
        # D2H), download u, p and dVddi.
        keep = []

        def pin(a):
            t = torch.from_numpy(a).pin_memory()
            keep.append(t)
            return t.numpy()

        hu, hq = pin(u.copy()), pin(q.copy())
        out_u, out_q, out_f = pin(A.real_field(p)), pin(A.real_field(p)), pin(A.real_field(p))
        E = np.array([0.0, 0.0, p.external_E_field[2]])
        e = fb.fg_energy()
        k_e2e = E2E_STEPS
        barrier()
        t0 = time.perf_counter()
        ctxm.set_state(hu, hq, 1.0, 0.0, H0)
        ctxm.mirror_force_mirror(e)
        for i in range(k_e2e):
            ctxm.set_uniform_E(E)
            ctxm.nose_poincare(e)
        strain = np.zeros(6)
        s_, pi_, h0_ = C.c_double(), C.c_double(), C.c_double()
        ctxm._check(A.lib().fg_get_state(ctxm._h, A.dptr(out_u), A.dptr(out_q), A.dptr(out_f), A.dptr(strain),
                                         C.byref(s_), C.byref(pi_), C.byref(h0_)))
        barrier()
        t1 = time.perf_counter()
        t_e2e = max_over_ranks(t1 - t0)
        field_bytes = u.nbytes
        e2e = {"value": p.N * k_e2e * world / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": (2 * field_bytes + 24 * k_e2e) / k_e2e,
               "d2h_bytes_per_step": (3 * field_bytes + 48 + C.sizeof(A.fg_energy) * k_e2e) / k_e2e,
               "steps": k_e2e, "includes": "fg_set_state + fg_mirror_force_mirror + K x (fg_set_uniform_E, "
                                           "fg_nose_poincare) + fg_get_state"}

    batched = None
    if rank == 0 and world == 1 and not args.no_batched and not args.mixed_only:
        batched = batched_sweep()
    fftc = epit = wstart = None
    if rank == 0 and world == 1 and not args.no_extras and not args.mixed_only:
        fftc = fft_vs_cufft(L)
        epit = epit_hysteresis()
        wstart = warm_start_leg(log=lambda m: print(m, file=sys.stderr, flush=True))
    sweep = points = None
    say = lambda m: print(m, file=sys.stderr, flush=True)
    if rank == 0 and world == 1 and not args.no_batched and not args.mixed_only:
        sweep = chained_sweep(n_points=args.sweep_points, log=say)
        points = parallel_points(warm_layers=wstart.pop("_layers", None) if wstart else None, log=say)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(p)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (fields, FFT, forces); f64 thermostat, strain, energy sums",
        "data": "synthetic: uni64-seeded dipoles (sigma 0.03 A), BaTiO3 ZVR parameters",
        "config": bench_config(L, p.N, world),
        "fp64": {"value": value64, "ms_per_step": (ms_fp64 / steps64) if ms_fp64 else None, "steps": steps64},
        "mixed_over_fp64": (value / value64) if value64 else None,
        "force_err_mixed_vs_fp64": ferr,
        "force_err_16_configs": ferr16,
        "roofline": roofline, "step_roofline": step_roofline, "kernels": per_kernel,
        "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks, "batched": batched,
        "fft_vs_cufft": fftc, "epit_hysteresis": epit, "warm_start": wstart, "cooling_sweep": sweep,
        "parallel_points": points,
        "gpu_launches": A.FG_NPROF * args.steps,  # kernels per bulk NP step graph
    }
    ctxm.close()
    if ctx64 is not None:
        ctx64.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
