"""The C-ABI library loads and exports every symbol include/feram_gpu.h declares.
No device calls (runs without a GPU)."""
import ctypes as C
import os

import pytest

from feram_b200 import _capi as A


def test_library_is_in_tree_and_loads(fg):
    L = A.lib()
    assert os.path.dirname(L._name) == os.path.dirname(os.path.abspath(A.__file__))


def test_every_declared_symbol_is_exported(fg):
    L = A.lib()
    names = A.exported_symbols()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_sizes_match_header(fg):
    # fg_energy: 13 doubles; fg_average: fg_energy + 2 + 6 + 3 + 6 + 3 + 6 doubles + int (padded)
    assert C.sizeof(A.fg_energy) == 13 * 8
    assert C.sizeof(A.fg_average) == (13 + 2 + 6 + 3 + 6 + 3 + 6) * 8 + 8


def test_host_functions_need_no_device(fg):
    p = fg.default_params()
    assert (p.Lx, p.Ly, p.Lz, p.padding_y) == (32, 32, 32, 1)
    assert p.Q_Nose == 0.1 and p.seed[0] == 123456789 and p.seed[1] == 987654321
    out = (C.c_double * 3)()
    amp = (C.c_double * 3)(1.0, 2.0, 3.0)
    assert A.lib().fg_wave(A.FG_WAVE_NONE, 5, 0, 0, amp, out) == 0
    assert list(out) == [1.0, 2.0, 3.0]


def test_oracle_loads(oracle):
    for n in ("oracle_create", "oracle_force", "oracle_nose_poincare", "oracle_leapfrog", "oracle_uni64"):
        assert hasattr(oracle, n)


def test_profile_names_match_header_count(fg):
    """fg_profile_name names FG_NPROF kernels (the bulk step graph) and
    returns "" past them; the Python constant mirrors the header's."""
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "feram_gpu.h")).read()
    n = int(hdr.split("#define FG_NPROF")[1].split()[0])
    assert n == A.FG_NPROF
    L = A.lib()
    names = [L.fg_profile_name(i).decode() for i in range(n + 1)]
    assert all(names[:n]) and names[n] == ""
    assert names[0].startswith("k_kick_drift") and names[-2].startswith("k_assemble")
