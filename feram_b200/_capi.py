"""ctypes mirror of include/feram_gpu.h.

The structs below follow the C declarations member by member; the
library path resolution loads the in-tree ``libferam_gpu.so`` built by
``feram_b200/build.py``.  Nothing here falls back to Python arithmetic: a
missing library raises ``OSError`` at load time.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

RELAXOR_MAX = 3
FILENAME_LEN = 300

FG_OK, FG_ERR_ARG, FG_ERR_CUDA, FG_ERR_NAN, FG_ERR_TIMEOUT, FG_ERR_UNSUPPORTED, FG_ERR_IO, FG_ERR_STATE = range(8)
FG_BULK, FG_FILM, FG_EPIT, FG_E110 = range(4)
FG_NPROF = 5  # kernels of one Nose-Poincare step in fg_profile_step
FG_SAMPLE_COLS, FG_SAMPLE_CAP = 16, 8192  # sample series rows (fg_sample)
FG_METHOD_MD, FG_METHOD_VS, FG_METHOD_LF, FG_METHOD_HL = range(4)
(FG_WAVE_NONE, FG_WAVE_TRIANGULAR_COS, FG_WAVE_TRIANGULAR_SIN,
 FG_WAVE_RAMPING_ON, FG_WAVE_RAMPING_OFF, FG_WAVE_OTHER) = range(6)
FG_PREC_FP64, FG_PREC_MIXED = 0, 1

_D3 = C.c_double * RELAXOR_MAX


class fg_params(C.Structure):
    _fields_ = [
        ("method", C.c_int), ("continue_run", C.c_int),
        ("GPa", C.c_double * 3), ("kelvin", C.c_double),
        ("mass_dipo", _D3), ("mass_acou", _D3), ("Q_Nose", C.c_double),
        ("bulk_or_film", C.c_int), ("Lx", C.c_int), ("Ly", C.c_int), ("Lz", C.c_int),
        ("gap_id", C.c_int), ("padding_y", C.c_int), ("gap_dipole_u", C.c_double * 3),
        ("a0", C.c_double), ("epi_strain", C.c_double),
        ("dt", C.c_double), ("n_thermalize", C.c_int), ("n_average", C.c_int),
        ("n_E_wave_period", C.c_int), ("n_coord_freq", C.c_int), ("n_hl_freq", C.c_int),
        ("n_hysteresis_loop_continue", C.c_int),
        ("external_E_field", C.c_double * 3), ("E_wave_type", C.c_int),
        ("P_kappa2", _D3), ("P_alpha", _D3), ("P_gamma", _D3),
        ("P_k1", _D3), ("P_k2", _D3), ("P_k3", _D3), ("P_k4", _D3),
        ("j", C.c_double * 7),
        ("B11", C.c_double), ("B12", C.c_double), ("B44", C.c_double),
        ("B1xx", C.c_double), ("B1yy", C.c_double), ("B4yz", C.c_double),
        ("modulation_constant", C.c_double),
        ("seed", C.c_int * 2), ("init_dipo_avg", C.c_double * 3),
        ("init_dipo_dev", C.c_double * 3), ("k_stripe", C.c_double * 3),
        ("Z_star", _D3), ("epsilon_inf", C.c_double), ("kappa", C.c_double),
        ("plot_dispersion", C.c_int), ("output_polarization", C.c_int),
        ("delta_e", C.c_double), ("delta_e_acou", C.c_double), ("verbose", C.c_int),
        ("coord_directory", C.c_char * FILENAME_LEN),
        ("slice_directory", C.c_char * FILENAME_LEN),
        ("distribution_directory", C.c_char * FILENAME_LEN),
        ("filename", C.c_char * FILENAME_LEN),
        ("N", C.c_int), ("Ninv", C.c_double), ("dt_2", C.c_double),
        ("n_freedom", C.c_int), ("unit_cell_volume", C.c_double),
        ("pNa03", C.c_double * 3), ("temperature_eV", C.c_double),
        ("target_kinetic_energy", C.c_double), ("E_field_always_zero", C.c_int),
    ]


ENERGY_FIELDS = ["acou_kinetic", "dipo_kinetic", "short_range", "long_range",
                 "dipole_E_field", "unharmonic", "homo_strain", "homo_coupling",
                 "inho_strain", "inho_coupling", "inho_modulation", "total",
                 "H_Nose_Poincare"]
POTENTIAL_FIELDS = ENERGY_FIELDS[2:11]


class fg_energy(C.Structure):
    _fields_ = [(n, C.c_double) for n in ENERGY_FIELDS]

    def as_dict(self):
        return {n: getattr(self, n) for n in ENERGY_FIELDS}


class fg_average(C.Structure):
    _fields_ = [("energy", fg_energy), ("e2", C.c_double), ("dipo_kinetic_true", C.c_double),
                ("strain", C.c_double * 6), ("u", C.c_double * 3), ("uu", C.c_double * 6),
                ("p", C.c_double * 3), ("pp", C.c_double * 6), ("n_steps", C.c_int)]


def dptr(a: np.ndarray):
    """double* of a C-contiguous float64 array (or None)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "need contiguous float64"
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ---- reference layouts (coord_module.F:91-93) --------------------------------

def real_field(p, nc: int = 3) -> np.ndarray:
    """Zeroed padded real field in the reference's layout; numpy shape
    (Lz, Ly+padding_y, 2*(Lx/2+1), nc) is the C view of Fortran (nc, x, y, z)."""
    return np.zeros((p.Lz, p.Ly + p.padding_y, 2 * (p.Lx // 2 + 1), nc), dtype=np.float64)


def complex_field(p, nc: int = 3) -> np.ndarray:
    """Zeroed complex field, shape (Lz, Ly+padding_y, Lx/2+1, nc) complex128."""
    return np.zeros((p.Lz, p.Ly + p.padding_y, p.Lx // 2 + 1, nc), dtype=np.complex128)


def k_table(p, ncol: int = 3) -> np.ndarray:
    """(3, ncol, k) real table, shape (Lz, Ly+padding_y, Lx/2+1, ncol, 3)."""
    return np.zeros((p.Lz, p.Ly + p.padding_y, p.Lx // 2 + 1, ncol, 3), dtype=np.float64)


def physical(a: np.ndarray, p) -> np.ndarray:
    """View of the physical sites (z, y, x, comp) of a padded real field."""
    return a[:, :p.Ly, :p.Lx, :]


_HERE = os.path.dirname(os.path.abspath(__file__))
# FERAM_B200_LIB=checked selects the bounds-checked build of the same sources
LIB_PATH = os.path.join(_HERE, "libferam_gpu_checked.so" if os.environ.get("FERAM_B200_LIB") == "checked"
                        else "libferam_gpu.so")
_lib = None


def lib() -> C.CDLL:
    """Load the in-tree C-ABI library (built by feram_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: run `python feram_b200/build.py` "
                      "(there is no CPU fallback for the MD step)")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    dp = P(C.c_double)
    fp = P(C.c_float)
    vp = C.c_void_p
    sig = {
        "fg_default_param": (None, [P(fg_params)]),
        "fg_read_param": (C.c_int, [C.c_char_p, P(fg_params), C.c_char_p, C.c_int]),
        "fg_make_param": (C.c_int, [P(fg_params), C.c_char_p, C.c_int]),
        "fg_wave": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, dp, dp]),
        "fg_uni64_seed": (C.c_double, [C.c_int, C.c_int]),
        "fg_uni64": (C.c_double, []),
        "fg_normal_dist_seed": (C.c_double, [C.c_int, C.c_int]),
        "fg_normal_dist": (C.c_double, [C.c_double, C.c_double]),
        "fg_init_dipoR_host": (C.c_int, [P(fg_params), dp, dp]),
        "fg_create": (C.c_int, [P(fg_params), C.c_int, P(vp)]),
        "fg_destroy": (None, [vp]),
        "fg_last_error": (C.c_char_p, [vp]),
        "fg_stream": (vp, [vp]),
        "fg_build_tables": (C.c_int, [vp]),
        "fg_upload_tables": (C.c_int, [vp, dp, dp]),
        "fg_upload_modulation": (C.c_int, [vp, dp]),
        "fg_set_modulation_R": (C.c_int, [vp, dp]),
        "fg_get_long_range": (C.c_int, [vp, dp]),
        "fg_fft_r2c3": (C.c_int, [vp, dp, dp]),
        "fg_fft_c2r3": (C.c_int, [vp, dp, dp]),
        "fg_time_fft": (C.c_int, [vp, C.c_int, dp]),
        "fg_get_params": (C.c_int, [vp, C.POINTER(fg_params)]),
        "fg_chain_point": (C.c_int, [vp, C.c_double, dp, C.POINTER(fg_energy)]),
        "fg_write_coord": (C.c_int, [vp, C.c_char_p, C.c_int]),
        "fg_set_wave": (C.c_int, [vp, C.c_int, C.c_int]),
        "fg_batch_set_grouping": (C.c_int, [vp, C.c_int]),
        "fg_batch_groups": (C.c_int, [vp]),
        "fg_batch_set_priorities": (C.c_int, [vp, C.c_int]),
        "fg_sample": (C.c_int, [vp]),
        "fg_samples_read": (C.c_int, [vp, dp, C.c_int, P(C.c_int)]),
        "fg_run_point": (C.c_int, [vp, C.c_double, dp, C.c_int, C.c_int, C.c_int, C.POINTER(fg_energy)]),
        "fg_batch_run_point": (C.c_int, [vp, dp, dp, C.c_int, C.c_int, C.c_int]),
        "fg_tune": (C.c_int, [vp, C.c_int, P(C.c_int), P(C.c_int), dp]),
        "fg_batch_tune": (C.c_int, [vp, C.c_int, dp, dp]),
        "fg_set_plan": (C.c_int, [vp, C.c_int, C.c_int]),
        "fg_get_plan": (C.c_int, [vp, P(C.c_int), P(C.c_int), P(C.c_int), P(C.c_int)]),
        "fg_wisdom_export": (C.c_int, [C.c_char_p, C.c_int, P(C.c_int)]),
        "fg_wisdom_import": (C.c_int, [C.c_char_p, P(C.c_int)]),
        "fg_wisdom_forget": (None, []),
        "fg_wisdom_measure": (C.c_int, [P(fg_params), C.c_int, C.c_int, C.c_char_p, C.c_int]),
        "fg_apply_wisdom": (C.c_int, [vp]),
        "fg_batch_apply_wisdom": (C.c_int, [vp]),
        "fg_ws_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.POINTER(vp)]),
        "fg_ws_destroy": (None, [vp]),
        "fg_ws_last_error": (C.c_char_p, [vp]),
        "fg_ws_forward": (C.c_int, [vp, fp, C.POINTER(C.c_ulonglong), fp]),
        "fg_ws_backward": (C.c_int, [vp, fp, C.POINTER(C.c_ulonglong), fp, fp, fp]),
        "fg_ws_backward_du": (C.c_int, [vp, fp, C.POINTER(C.c_ulonglong), fp, fp, fp, fp]),
        "fg_ws_adam": (C.c_int, [vp, C.c_float]),
        "fg_ws_layer_shape": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "fg_ws_get_layer": (C.c_int, [vp, C.c_int, fp, fp, fp, fp]),
        "fg_ws_set_layer": (C.c_int, [vp, C.c_int, fp, fp]),
        "fg_ws_get_io": (C.c_int, [vp, fp, fp]),
        "fg_ws_field": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "fg_set_state": (C.c_int, [vp, dp, dp, C.c_double, C.c_double, C.c_double]),
        "fg_get_state": (C.c_int, [vp, dp, dp, dp, dp, dp, dp, dp]),
        "fg_set_thermostat": (C.c_int, [vp, C.c_double, C.c_double, C.c_double]),
        "fg_get_acouK": (C.c_int, [vp, dp]),
        "fg_set_acou": (C.c_int, [vp, dp, dp]),
        "fg_upload_site_arrays": (C.c_int, [vp, dp, dp, dp, P(C.c_int), P(C.c_int), dp]),
        "fg_get_acou": (C.c_int, [vp, dp, dp, dp]),
        "fg_set_uniform_E": (C.c_int, [vp, dp]),
        "fg_mirror_force_mirror": (C.c_int, [vp, P(fg_energy)]),
        "fg_nose_poincare": (C.c_int, [vp, P(fg_energy)]),
        "fg_leapfrog": (C.c_int, [vp, P(fg_energy), C.c_int]),
        "fg_kinetic_energy_dipo": (C.c_int, [vp, dp]),
        "fg_velocity_scaling": (C.c_int, [vp, P(fg_energy)]),
        "fg_batch_create": (C.c_int, [C.c_int, P(fg_params), C.c_int, P(vp), C.c_char_p, C.c_int]),
        "fg_batch_destroy": (None, [vp]),
        "fg_batch_size": (C.c_int, [vp]),
        "fg_batch_context": (vp, [vp, C.c_int]),
        "fg_batch_last_error": (C.c_char_p, [vp]),
        "fg_batch_step": (C.c_int, [vp, C.c_int, P(fg_energy)]),
        "fg_nose_poincare_hamiltonian": (C.c_int, [vp, P(fg_energy)]),
        "fg_average_accumulate": (C.c_int, [vp, P(fg_energy), P(fg_average)]),
        "fg_dipoRavg_accumulate": (C.c_int, [vp]),
        "fg_get_dipoRavg": (C.c_int, [vp, dp]),
        "fg_run_steps": (C.c_int, [vp, C.c_int, P(fg_energy)]),
        "fg_time_steps": (C.c_int, [vp, C.c_int, dp]),
        "fg_profile_step": (C.c_int, [vp, C.c_int, dp]),
        "fg_profile_name": (C.c_char_p, [C.c_int]),
        "fg_feram_run": (C.c_int, [C.c_char_p, C.c_int, P(fg_average), dp, C.c_char_p, C.c_int]),
        "fg_kinetic_energy_dipo_noalloc": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, dp, P(C.c_ubyte), vp, vp,
                                                     C.c_char_p, C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name, None)
        if f is None:
            continue
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Names declared in include/feram_gpu.h (used by the export test)."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "feram_gpu.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(fg_[A-Za-z0-9_]+)\s*\(", text)))
