"""ctypes view of the FP64 CPU oracle (oracle/liboracle.so) for the tests.

The oracle is the checker: tests call it on the same inputs as the device
path and compare.  It is built from oracle/Makefile when missing.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from feram_b200 import _capi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "liboracle.so")
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    L = C.CDLL(LIB)
    P, dp, vp = C.POINTER, C.POINTER(C.c_double), C.c_void_p
    sig = {
        "oracle_create": (vp, [P(A.fg_params), C.c_char_p, C.c_int]),
        "oracle_destroy": (None, [vp]),
        "oracle_get_tables": (C.c_int, [vp, dp, dp]),
        "oracle_get_inhomo_tables": (C.c_int, [vp, dp, dp, dp]),
        "oracle_set_modulation_R": (C.c_int, [vp, dp]),
        "oracle_get_modulation": (C.c_int, [vp, dp]),
        "oracle_set_state": (C.c_int, [vp, dp, dp, C.c_double, C.c_double, C.c_double]),
        "oracle_get_state": (C.c_int, [vp, dp, dp, dp, dp, dp, dp, dp]),
        "oracle_get_acouK": (C.c_int, [vp, dp]),
        "oracle_set_acou": (C.c_int, [vp, dp, dp]),
        "oracle_set_sites": (C.c_int, [vp, dp, dp, dp, P(C.c_int), P(C.c_int), dp]),
        "oracle_get_acou": (C.c_int, [vp, dp, dp, dp]),
        "oracle_acouR_for_coord": (C.c_int, [vp, dp]),
        "oracle_set_uniform_E": (C.c_int, [vp, dp]),
        "oracle_force": (C.c_int, [vp, P(A.fg_energy)]),
        "oracle_nose_poincare": (C.c_int, [vp, P(A.fg_energy)]),
        "oracle_leapfrog": (C.c_int, [vp, P(A.fg_energy), C.c_int]),
        "oracle_velocity_scaling": (C.c_int, [vp, P(A.fg_energy)]),
        "oracle_kinetic_energy_dipo": (C.c_double, [vp]),
        "oracle_nose_poincare_hamiltonian": (C.c_double, [vp, P(A.fg_energy)]),
        "oracle_initialize": (C.c_int, [vp, P(A.fg_energy)]),
        "oracle_md": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, P(A.fg_energy), P(A.fg_average)]),
        "oracle_average_accumulate": (C.c_int, [vp, P(A.fg_energy), P(A.fg_average)]),
        "oracle_uni64_seed": (C.c_double, [C.c_int, C.c_int]),
        "oracle_uni64": (C.c_double, []),
        "oracle_normal_dist_seed": (C.c_double, [C.c_int, C.c_int]),
        "oracle_normal_dist": (C.c_double, [C.c_double, C.c_double]),
        "oracle_wave": (None, [C.c_int, C.c_int, C.c_int, C.c_int, dp, dp]),
        "oracle_r2c": (C.c_int, [C.c_int] * 5 + [dp, dp]),
        "oracle_c2r": (C.c_int, [C.c_int] * 5 + [dp, dp]),
        "oracle_set_threads": (None, [C.c_int]),
        "oracle_default_param": (None, [P(A.fg_params)]),
        "oracle_make_param": (C.c_int, [P(A.fg_params)]),
        "oracle_init_dipoR": (C.c_int, [P(A.fg_params), dp, dp]),
    }
    for n, (r, a) in sig.items():
        f = getattr(L, n)
        f.restype = r
        f.argtypes = a
    _lib = L
    return L


class Oracle:
    """One oracle supercell (mirror of feram_b200.Context's methods)."""

    def __init__(self, p):
        self.L = load()
        self.p = p
        eb = C.create_string_buffer(400)
        self.h = self.L.oracle_create(C.byref(p), eb, 400)
        if not self.h:
            raise RuntimeError(eb.value.decode())

    def close(self):
        if self.h:
            self.L.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tables(self):
        sr, lr = A.k_table(self.p), A.k_table(self.p)
        self.L.oracle_get_tables(self.h, A.dptr(sr), A.dptr(lr))
        return sr, lr

    def set_modulation_R(self, modR):
        self.L.oracle_set_modulation_R(self.h, A.dptr(modR))

    def modulation(self):
        c = A.complex_field(self.p)
        self.L.oracle_get_modulation(self.h, A.dptr(c.view(np.float64)))
        return c

    def set_state(self, dipoR=None, dipoP=None, s=1.0, pi=0.0, H0=0.0):
        self.L.oracle_set_state(self.h, A.dptr(dipoR), A.dptr(dipoP), s, pi, H0)

    def get_state(self):
        u, q, f = A.real_field(self.p), A.real_field(self.p), A.real_field(self.p)
        strain = np.zeros(6)
        s, pi, H0 = C.c_double(), C.c_double(), C.c_double()
        self.L.oracle_get_state(self.h, A.dptr(u), A.dptr(q), A.dptr(f), A.dptr(strain),
                                C.byref(s), C.byref(pi), C.byref(H0))
        return dict(dipoR=u, dipoP=q, dVddi=f, strain=strain, s=s.value, pi=pi.value, H0=H0.value)

    def acouK(self):
        a = A.complex_field(self.p)
        self.L.oracle_get_acouK(self.h, A.dptr(a.view(np.float64)))
        return a

    def set_sites(self, Z_starR=None, mass_dipo_inv=None, mass_acou_inv=None, relaxor=None, sum_p=None,
                  E_field_local=None):
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None
        dp_ = lambda a: A.dptr(a) if a is not None else None
        self.L.oracle_set_sites(self.h, dp_(Z_starR), dp_(mass_dipo_inv), dp_(mass_acou_inv), ip(relaxor),
                                ip(sum_p), dp_(E_field_local))

    def set_acou(self, acouR=None, acouP=None):
        self.L.oracle_set_acou(self.h, A.dptr(acouR) if acouR is not None else None,
                               A.dptr(acouP) if acouP is not None else None)

    def get_acou(self):
        r, q, d = A.real_field(self.p), A.real_field(self.p), A.real_field(self.p)
        self.L.oracle_get_acou(self.h, A.dptr(r), A.dptr(q), A.dptr(d))
        return {"acouR": r, "acouP": q, "dVdacR": d}

    def acouR_for_coord(self):
        a = A.real_field(self.p)
        self.L.oracle_acouR_for_coord(self.h, A.dptr(a))
        return a

    def set_uniform_E(self, E):
        e = np.ascontiguousarray(E, dtype=np.float64)
        self.L.oracle_set_uniform_E(self.h, A.dptr(e))

    def force(self, e=None):
        e = e if e is not None else A.fg_energy()
        self.L.oracle_force(self.h, C.byref(e))
        return e

    def nose_poincare(self, e):
        self.L.oracle_nose_poincare(self.h, C.byref(e))
        return e

    def leapfrog(self, e, i_step):
        self.L.oracle_leapfrog(self.h, C.byref(e), i_step)
        return e

    def velocity_scaling(self, e):
        self.L.oracle_velocity_scaling(self.h, C.byref(e))
        return e

    def kinetic_energy_dipo(self):
        return self.L.oracle_kinetic_energy_dipo(self.h)

    def initialize(self):
        e = A.fg_energy()
        self.L.oracle_initialize(self.h, C.byref(e))
        return e

    def md(self, i_first, i_last, set_H0, e, avg=None):
        rc = self.L.oracle_md(self.h, i_first, i_last, set_H0, C.byref(e), C.byref(avg) if avg is not None else None)
        assert rc == 0, rc
        return e


def r2c(field, p, nc=3):
    out = np.zeros((p.Lz, p.Ly + p.padding_y, p.Lx // 2 + 1, nc), dtype=np.complex128)
    load().oracle_r2c(p.Lx, p.Ly, p.Lz, p.padding_y, nc, A.dptr(np.ascontiguousarray(field)),
                      A.dptr(out.view(np.float64)))
    return out
