"""The oracle (and the host-side restatements the product shares the
arithmetic of) against the reference's own known answers."""
import ctypes as C

import numpy as np
import pytest

import helpers
import oracle_lib
from feram_b200 import _capi as A


def _kat_check(seed, nxt):
    k = helpers.golden("uni64_kat.json")
    assert seed(*k["seed"]) >= 1.0
    for _ in range(k["skip"]):
        nxt()
    got = [nxt() * 9007199254740992.0 for _ in range(5)]
    assert got == [float(v) for v in k["next_times_2p53"]]


def test_uni64_kat_oracle(oracle):
    _kat_check(oracle.oracle_uni64_seed, oracle.oracle_uni64)


def test_uni64_kat_product_host(fg):
    L = A.lib()
    _kat_check(L.fg_uni64_seed, L.fg_uni64)


def test_uni64_seed_return_counts(fg):
    # marsaglia_tsang_uni64_check.F: successive seedings return 1.0, 2.0, ...
    L = A.lib()
    a = L.fg_uni64_seed(1, 2)
    b = L.fg_normal_dist_seed(3, 4)
    assert b == a + 1.0


@pytest.mark.parametrize("which", ["oracle", "product"])
def test_wave_kat(which, oracle, fg):
    k = helpers.golden("wave_kat.json")
    codes = {"triangular_cos": A.FG_WAVE_TRIANGULAR_COS, "triangular_sin": A.FG_WAVE_TRIANGULAR_SIN,
             "ramping_on": A.FG_WAVE_RAMPING_ON, "ramping_off": A.FG_WAVE_RAMPING_OFF}
    amp = (C.c_double * 3)(*k["amplitude"])
    for c in k["cases"]:
        out = (C.c_double * 3)()
        if which == "oracle":
            oracle.oracle_wave(codes[c["type"]], int(c["i_step"]), k["n_thermalize"], k["period"], amp, out)
        else:
            assert A.lib().fg_wave(codes[c["type"]], int(c["i_step"]), k["n_thermalize"], k["period"], amp, out) == 0
        assert out[c["comp"]] == c["expect"], c


@pytest.mark.parametrize("shape", [(12, 10, 6), (16, 16, 16), (8, 15, 9)])
def test_oracle_fft_matches_numpy(shape, oracle):
    Lx, Ly, Lz = shape
    pad, nc = 1, 3
    rng = np.random.default_rng(7)
    a = np.zeros((Lz, Ly + pad, 2 * (Lx // 2 + 1), nc))
    a[:, :Ly, :Lx] = rng.standard_normal((Lz, Ly, Lx, nc))
    out = np.zeros((Lz, Ly + pad, Lx // 2 + 1, nc), dtype=np.complex128)
    oracle.oracle_r2c(Lx, Ly, Lz, pad, nc, A.dptr(a), A.dptr(out.view(np.float64)))
    ref = np.fft.rfftn(a[:, :Ly, :Lx], axes=(0, 1, 2))
    assert np.abs(out[:, :Ly] - ref).max() <= 1e-13 * np.abs(ref).max()
    # c2r of a non-Hermitian half spectrum: FFTW's half-complex projection
    X = rng.standard_normal(out.shape) + 1j * rng.standard_normal(out.shape)
    back = np.zeros_like(a)
    Xc = X.copy()
    oracle.oracle_c2r(Lx, Ly, Lz, pad, nc, A.dptr(Xc.view(np.float64)), A.dptr(back))
    refb = np.fft.irfftn(X[:, :Ly], s=(Lz, Ly, Lx), axes=(0, 1, 2)) * (Lx * Ly * Lz)
    assert np.abs(back[:, :Ly, :Lx] - refb).max() <= 1e-13 * np.abs(refb).max()


def fortran_E(v, d=6):
    """Fortran Ew.d mantissa form 0.dddddd E+xx (no padding)."""
    import math
    if v == 0:
        return "0." + "0" * d + "E+00"
    e = math.floor(math.log10(abs(v))) + 1
    s = "%.*f" % (d, abs(v) / 10 ** e)
    if s.startswith("1."):
        e += 1
        s = "%.*f" % (d, abs(v) / 10 ** e)
    return ("-" if v < 0 else "") + s + "E%+03d" % e


def modulation_setup(p):
    k = helpers.golden("modulation_kat.json")
    mod = np.zeros((p.Lz, p.Ly + p.padding_y, 2 * (p.Lx // 2 + 1)))
    for ix, iy, iz, v in k["modulation"]:
        mod[int(iz), int(iy), int(ix)] = v
    return k, mod


def test_modulation_check_kat_oracle(fg):
    """modulation_check.sh:64-79 on the oracle: 3 log lines of each energy and
    six acoustic vectors of each sign."""
    k = helpers.golden("modulation_kat.json")
    p = fg.params_from_text(k["feram"], "zzzmodulation")
    _, mod = modulation_setup(p)
    o = oracle_lib.Oracle(p)
    o.set_modulation_R(mod)
    e = o.initialize()
    lines = []
    lines.append(e.inho_strain / p.N)
    mods = [e.inho_modulation / p.N]
    for i in (1, 2):
        o.leapfrog(e, i)
        lines.append(e.inho_strain / p.N)
        mods.append(e.inho_modulation / p.N)
    assert ["%.12f" % v for v in lines] == [k["inho_strain_per_cell"]] * k["n_log_lines"]
    assert ["%.12f" % v for v in mods] == [k["inho_modulation_per_cell"]] * k["n_log_lines"]
    # the .coord of step 1 (n_coord_freq = 1) is written after step 1; acouR
    # depends only on u (= 0 here), so the current state gives the same vectors
    ac = A.physical(o.acouR_for_coord(), p).ravel()
    vals = [fortran_E(v) for v in ac]
    assert vals.count(k["acouR_abs"]) == k["n_vectors_each_sign"]
    assert vals.count("-" + k["acouR_abs"]) == k["n_vectors_each_sign"]


def test_long_range_dispersion_golden_oracle(fg):
    g = helpers.golden("dispersion_long64.json")
    p = fg.default_params()
    p.Lx, p.Ly, p.Lz = g["L"]
    p.a0 = g["a0"]
    p.Z_star[0] = g["Z_star"]
    p.epsilon_inf = g["epsilon_inf"]
    fg.make_param(p)
    o = oracle_lib.Oracle(p)
    _, lr = o.tables()
    scale = 0.0
    worst = 0.0
    for pt in g["points"]:
        ix, iy, iz = pt["k"]
        M = p.Z_star[0] ** 2 * lr[iz, iy, ix]
        scale = max(scale, np.abs(M).max())
        # printed 3x3 matrix, 6 significant digits
        assert np.allclose(M, np.array(pt["matrix"]), rtol=1e-5, atol=1e-6 * 34)
        if (ix, iy, iz) != (0, 0, 0):  # the reference's eigenvalue line at Gamma disagrees with its own matrix
            worst = max(worst, np.abs(np.sort(np.linalg.eigvalsh(M)) - np.sort(pt["eig"])).max())
    assert worst <= 1e-12 * scale, worst


def short_range_analytic(p, kx, ky, kz):
    """numpy restatement of the 27-point stencil's transform (same formula as
    the device kernel's short_range_k)."""
    th = [2 * np.pi * kx / p.Lx, 2 * np.pi * ky / p.Ly, 2 * np.pi * kz / p.Lz]
    c = [np.cos(t) for t in th]
    s = [np.sin(t) for t in th]
    j = list(p.j)
    S = np.zeros((3, 3))
    for a in range(3):
        b, g = (a + 1) % 3, (a + 2) % 3
        S[a, a] = (2 * p.P_kappa2[0] + 2 * j[1] * c[a] + 2 * j[0] * (c[b] + c[g]) + 4 * j[3] * c[b] * c[g]
                   + 4 * j[2] * c[a] * (c[b] + c[g]) + 8 * j[5] * c[0] * c[1] * c[2])
    for a, b, g in ((1, 2, 0), (2, 0, 1), (0, 1, 2)):
        S[a, b] = S[b, a] = -4 * j[4] * s[a] * s[b] - 8 * j[6] * s[a] * s[b] * c[g]
    return S


def test_short_range_analytic_matches_oracle_fft(fg):
    p = helpers.params(L="12 10 8")
    o = oracle_lib.Oracle(p)
    sr, _ = o.tables()
    worst = 0.0
    for kz in range(p.Lz):
        for ky in range(p.Ly):
            for kx in range(p.Lx // 2 + 1):
                worst = max(worst, np.abs(sr[kz, ky, kx] - short_range_analytic(p, kx, ky, kz)).max())
    assert worst <= 1e-13 * np.abs(sr).max()


def test_initial_dipoles_bit_exact(fg):
    """initialize_dipoR's seeded Gaussian u: product host == oracle, bitwise."""
    p = helpers.params(L="8 6 4", init_dipo_avg="0.01 0.02 -0.03", init_dipo_dev="0.05 0.04 0.03",
                       k_stripe="0.0 0.0 0.25")
    u = A.real_field(p)
    assert A.lib().fg_init_dipoR_host(C.byref(p), A.dptr(u), None) == 0
    o = oracle_lib.Oracle(p)
    o.initialize()
    uo = o.get_state()["dipoR"]
    assert np.array_equal(A.physical(u, p), A.physical(uo, p))


def test_oracle_nose_poincare_is_second_order(fg):
    """Bond-Leimkuhler-Laird NP is symplectic and second order: the excursion
    of H_NP over a fixed time window scales as dt^2."""
    peaks = []
    for dt in (0.002, 0.001):
        p = helpers.params(L="8 8 8", kelvin="300", dt=str(dt))
        o = oracle_lib.Oracle(p)
        e = o.initialize()
        o.md(1, 0, 1, e)  # H0 from the initial state only
        h = 0.0
        for _ in range(int(round(0.08 / dt))):
            o.nose_poincare(e)
            h = max(h, abs(e.H_Nose_Poincare))
        peaks.append(h)
    assert 3.6 < peaks[0] / peaks[1] < 4.4, peaks


def test_oracle_velocity_scaling_hits_target_kinetic_energy(fg):
    """velocity_scaling.F:75-83: after the rescale the kinetic energy of the
    masked momenta equals target_kinetic_energy = 3/2 N k T."""
    p = helpers.params(L="8 8 8", method="'vs'", kelvin="250")
    o = oracle_lib.Oracle(p)
    o.set_state(helpers.seeded_u(p, 3, sigma=0.05), helpers.seeded_p(p, 3, sigma=0.01))
    e = o.force()
    for _ in range(3):
        o.velocity_scaling(e)
    assert abs(o.kinetic_energy_dipo() - p.target_kinetic_energy) <= 1e-12 * p.target_kinetic_energy
    assert e.dipo_kinetic > 0.0
