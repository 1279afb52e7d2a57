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


def test_sample_constants_match_header(fg):
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "feram_gpu.h")).read()
    assert int(hdr.split("#define FG_SAMPLE_COLS")[1].split()[0]) == A.FG_SAMPLE_COLS
    assert int(hdr.split("#define FG_SAMPLE_CAP")[1].split()[0]) == A.FG_SAMPLE_CAP


def test_wisdom_round_trip_needs_no_device(fg):
    """fg_wisdom_import / fg_wisdom_export: the text form round-trips, later
    plans replace earlier ones of the same key, and a malformed line imports
    nothing (as fftw_import_wisdom_from_filename fails as a whole)."""
    fg.wisdom_forget()
    try:
        assert fg.wisdom_export() == "feram_b200 wisdom 1\n"
        text = ("feram_b200 wisdom 1\n# a comment\nsolo mixed 128 128 128 9 8 1\n"
                "batch fp64 16 16 16 12 2 0\nbatch mixed 24 24 24 9 4 2\n")
        assert fg.wisdom_import(text) == 3
        out = fg.wisdom_export()
        lines = out.splitlines()
        assert lines[0] == "feram_b200 wisdom 1" and len(lines) == 4
        assert sorted(lines[1:]) == sorted(["solo mixed 128 128 128 9 8 1", "batch fp64 16 16 16 12 2 0",
                                            "batch mixed 24 24 24 9 4 2"])
        assert fg.wisdom_import("feram_b200 wisdom 1\nsolo mixed 128 128 128 9 4 0\n") == 1
        assert "solo mixed 128 128 128 9 4 0" in fg.wisdom_export().splitlines()
        before = fg.wisdom_export()
        for bad in ("solo mixed 8 8 8 9 4 1\n",                                   # no header
                    "feram_b200 wisdom 1\nsolo mixed 8 8 8 9 4\n",                # short line
                    "feram_b200 wisdom 1\nsolo half 8 8 8 9 4 1\n",               # unknown precision
                    "feram_b200 wisdom 1\nsolo mixed 8 8 8 9 -1 1\n",             # negative width
                    "feram_b200 wisdom 1\nsolo mixed 8 8 8 9 4 1\nsolo mixed 8 8 8 9 4 1 7\n"):
            with pytest.raises(fg.FeramError):
                fg.wisdom_import(bad)
        assert fg.wisdom_export() == before
        n = C.c_int()
        assert A.lib().fg_wisdom_export(None, 0, C.byref(n)) == 0 and n.value == len(before) + 1
        small = C.create_string_buffer(4)
        assert A.lib().fg_wisdom_export(small, 4, C.byref(n)) == A.FG_ERR_ARG
    finally:
        fg.wisdom_forget()
