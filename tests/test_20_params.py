"""The host-side .feram parser (read_Param / make_Param mirror)."""
import math

import numpy as np

import pytest

import helpers
from feram_b200 import _capi as A


def test_parse_zzznp(fg):
    p = fg.params_from_text(helpers.golden("zzznp.feram"), "zzznp")
    assert p.method == A.FG_METHOD_MD and p.bulk_or_film == A.FG_BULK
    assert list(p.GPa) == [-5.0] * 3  # one value -> hydrostatic
    assert (p.Lx, p.Ly, p.Lz) == (16, 16, 16)
    assert p.kelvin == 300 and p.temperature_eV == 300 / 11604.45
    assert p.mass_dipo[0] == 39.0 / 9648.53377163899 and p.mass_dipo[2] == p.mass_dipo[0]
    assert p.a0 == 3.94 and p.dt == 0.002
    assert list(p.j) == [-2.648, 3.894, 0.898, -0.789, 0.562, 0.358, 0.179]
    assert p.P_kappa2[0] == 5.502 and p.P_alpha[1] == 110.4 and p.P_gamma[2] == -163.1
    assert p.B11 == 126.0 and p.B1xx == -211.0 and p.B4yz == -7.75
    assert list(p.init_dipo_avg) == [0.143] * 3
    assert p.Z_star[0] == 9.956 and p.epsilon_inf == 5.24
    assert p.coord_directory == b"never"
    assert p.Q_Nose == 0.1 and p.padding_y == 1 and p.E_field_always_zero == 1
    # make_Param
    assert p.N == 4096 and p.n_freedom == 3 * 4096 and p.dt_2 == 0.001
    assert p.kappa == math.sqrt(math.pi) / 3.94 / 4096 ** (1 / 6)
    assert p.pNa03[0] == -5.0 * 0.01 / 1.60217653 * 4096 * (3.94 * 3.94 * 3.94)  # a0**3 as repeated products


def test_parse_zzz16_logical_typo_and_seed(fg):
    p = fg.params_from_text(helpers.golden("zzz16.feram"), "zzz16")
    assert p.output_polarization == 1  # '.ture.' reads as .true.
    assert list(p.seed) == [1242914819, 1957271591]
    assert p.Q_Nose == 0.05 and p.P_k4[0] == 641.968099408642


def test_parse_leapfrog_acoustic_mass(fg):
    p = fg.params_from_text(helpers.golden("zzzlf.feram"), "zzzlf")
    assert p.method == A.FG_METHOD_LF
    assert p.mass_acou[0] == 46.44 / 9648.53377163899


@pytest.mark.parametrize("bad,needle", [
    ("nonsense = 1", "No such parameter"),
    ("bulk_or_film = 'slab'", "bulk_or_film"),
    ("acoustic_mass_amu = 40.0", "togeter"),
    ("n_E_wave_period = 6", "divided by 4"),
])
def test_parse_errors(fg, bad, needle):
    with pytest.raises(fg.FeramError) as ei:
        fg.params_from_text("method = 'md'\n" + bad + "\n", "bad")
    assert needle in str(ei.value)


def test_make_param_gap_check(fg):
    with pytest.raises(fg.FeramError):
        fg.params_from_text("gap_id = 1\n", "bad")
    p = fg.params_from_text("bulk_or_film = 'epit'\nL = 8 8 7\ngap_id = 1\n", "ok")
    assert p.gap_id == 1


def _struct_bytes(p):
    import ctypes as C
    return bytes(C.string_at(C.addressof(p), C.sizeof(p)))


def test_oracle_defaults_match_product(fg, oracle):
    """read_Param's defaults restated twice (product host code and oracle)."""
    import ctypes as C
    a, b = A.fg_params(), A.fg_params()
    fg.lib().fg_default_param(C.byref(a))
    oracle.oracle_default_param(C.byref(b))
    assert _struct_bytes(a) == _struct_bytes(b)


@pytest.mark.parametrize("deck,tags", [
    ("zzznp.feram", {}),
    ("zzz16.feram", {}),
    ("zzznp.feram", dict(L="20 12 18", kelvin="450", GPa="-3 -4 -5")),
    ("zzznp.feram", dict(L="12 12 8", bulk_or_film="'epit'", epi_strain="0.01")),
])
def test_oracle_make_param_and_init_match_product(fg, oracle, deck, tags):
    """make_Param's derived constants and initialize_dipoR's uni64 draw:
    the oracle's own restatements give the product's values bit for bit, so
    a CPU run built from the oracle alone (the timed reference arm) has the
    inputs of the device run."""
    import ctypes as C
    p = helpers.params(deck, **tags)
    q = A.fg_params.from_buffer_copy(p)
    q.N = 0
    q.kappa = 0.0  # none of these decks sets kappa: make_Param derives it
    assert oracle.oracle_make_param(C.byref(q)) == 0
    assert _struct_bytes(p) == _struct_bytes(q)
    u1, q1 = A.real_field(p), A.real_field(p)
    u2, q2 = A.real_field(p), A.real_field(p)
    assert fg.lib().fg_init_dipoR_host(C.byref(p), A.dptr(u1), A.dptr(q1)) == 0
    assert oracle.oracle_init_dipoR(C.byref(p), A.dptr(u2), A.dptr(q2)) == 0
    assert np.array_equal(u1, u2) and np.array_equal(q1, q2)


def test_reference_arm_inputs_load_no_product_library():
    """bench.py --impl reference builds its parameters and initial state from
    the oracle alone: a fresh process doing so maps no product library."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys; sys.path.insert(0, %r); import bench, json; "
            "p = bench.make_params(16, impl='reference'); u, q = bench.initial_state(p, impl='reference'); "
            "print(json.dumps({'libs': bench.loaded_repo_libs(), 'N': p.N, 'u': float(abs(u).sum())}))" % root)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["libs"] == ["oracle/liboracle.so"], out
    assert out["N"] == 4096 and out["u"] > 0
