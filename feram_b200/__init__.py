"""feram_b200 -- B200-native MD step of feram's effective Hamiltonian.

The product is the C-ABI shared library ``libferam_gpu.so`` (declared in
``include/feram_gpu.h``).  This module is the Python view of that interface
for tests and benchmarks: ``Context`` wraps one ``fg_ctx`` and its methods
carry the names of the reference subroutines they replace
(``mirror_force_mirror``, ``nose_poincare``, ``leapfrog``,
``kinetic_energy_dipo`` ...).  Arrays are numpy views of the reference's
padded Fortran layout (see ``_capi.real_field``).  Every call goes to the
device; there is no CPU fallback, and a missing library raises ``OSError``.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

from . import _capi
from ._capi import (FG_PREC_FP64, FG_PREC_MIXED, FG_OK, FG_SAMPLE_COLS, fg_average, fg_energy, fg_params,
                    complex_field, dptr, k_table, physical, real_field)

__all__ = ["Context", "FeramError", "read_param", "make_param", "params_from_text", "default_params",
           "FG_PREC_FP64", "FG_PREC_MIXED", "fg_energy", "fg_average", "fg_params",
           "real_field", "complex_field", "k_table", "physical", "lib", "Batch",
           "wisdom_export", "wisdom_import", "wisdom_forget", "wisdom_measure", "FG_SAMPLE_COLS"]

lib = _capi.lib


class FeramError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _err(buf) -> str:
    return buf.value.decode(errors="replace")


def default_params() -> fg_params:
    p = fg_params()
    lib().fg_default_param(C.byref(p))
    return p


def read_param(path: str) -> fg_params:
    """read_Param (param_module.F:114-450) on the host."""
    p = fg_params()
    eb = C.create_string_buffer(512)
    rc = lib().fg_read_param(os.fsencode(path), C.byref(p), eb, 512)
    if rc:
        raise FeramError(rc, _err(eb))
    return p


def make_param(p: fg_params) -> fg_params:
    """make_Param (param_module.F:452-480), in place."""
    eb = C.create_string_buffer(512)
    rc = lib().fg_make_param(C.byref(p), eb, 512)
    if rc:
        raise FeramError(rc, _err(eb))
    return p


def params_from_text(text: str, name: str = "input") -> fg_params:
    """Parse .feram text (through a temporary file) and make the derived constants."""
    with tempfile.TemporaryDirectory() as d:
        fn = os.path.join(d, name + ".feram")
        with open(fn, "w") as f:
            f.write(text)
        p = read_param(fn)
    return make_param(p)


class Context:
    """One supercell on the current CUDA device (alloc_Coord + Coord_type)."""

    def __init__(self, params: fg_params, precision: int = FG_PREC_FP64):
        self.p = params
        self.precision = precision
        self._h = C.c_void_p()
        rc = lib().fg_create(C.byref(params), precision, C.byref(self._h))
        if rc:
            msg = self.last_error()
            self.close()
            raise FeramError(rc, msg)

    # -- plumbing
    def last_error(self) -> str:
        if not self._h:
            return "no context"
        r = lib().fg_last_error(self._h)
        return r.decode() if r else ""

    def _check(self, rc):
        if rc != FG_OK:
            raise FeramError(rc, self.last_error())

    def close(self):
        if self._h:
            lib().fg_destroy(self._h)
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

    @property
    def stream(self) -> int:
        return lib().fg_stream(self._h)

    # -- setup
    def build_tables(self):
        self._check(lib().fg_build_tables(self._h))

    def upload_tables(self, short_range: np.ndarray, long_range: np.ndarray):
        self._check(lib().fg_upload_tables(self._h, dptr(short_range), dptr(long_range)))

    def upload_modulation(self, c_k_modulation_k: np.ndarray | None):
        a = None if c_k_modulation_k is None else np.ascontiguousarray(c_k_modulation_k).view(np.float64)
        self._check(lib().fg_upload_modulation(self._h, dptr(a)))

    def set_modulation_R(self, modulation_R: np.ndarray):
        self._check(lib().fg_set_modulation_R(self._h, dptr(modulation_R)))

    def get_long_range(self) -> np.ndarray:
        t = k_table(self.p)
        self._check(lib().fg_get_long_range(self._h, dptr(t)))
        return t

    # -- FFTs (plan_r2c_3_out / plan_c2r_3_out)
    def fft_r2c3(self, field: np.ndarray) -> np.ndarray:
        out = complex_field(self.p)
        self._check(lib().fg_fft_r2c3(self._h, dptr(field), dptr(out.view(np.float64))))
        return out

    def fft_c2r3(self, spec: np.ndarray) -> np.ndarray:
        out = real_field(self.p)
        s = np.ascontiguousarray(spec, dtype=np.complex128)
        self._check(lib().fg_fft_c2r3(self._h, dptr(s.view(np.float64)), dptr(out)))
        return out

    def time_fft(self, reps: int = 20):
        """fg_time_fft: device milliseconds of the 3-component r2c and c2r."""
        ms = (C.c_double * 2)()
        self._check(lib().fg_time_fft(self._h, reps, ms))
        return ms[0], ms[1]

    def chain_point(self, kelvin: float, E=None) -> fg_energy:
        """fg_chain_point: the next sweep point from the state on the device
        (p / s, new kelvin and field, force, s = 1, pi = 0, H0)."""
        e = fg_energy()
        Ea = None if E is None else np.ascontiguousarray(E, dtype=np.float64)
        self._check(lib().fg_chain_point(self._h, kelvin, dptr(Ea), C.byref(e)))
        p = fg_params()
        self._check(lib().fg_get_params(self._h, C.byref(p)))
        self.p = p
        return e

    def set_wave(self, on: bool = True, i_step: int = 0):
        """fg_set_wave: the per-step field wave() evaluated on the device."""
        self._check(lib().fg_set_wave(self._h, 1 if on else 0, i_step))

    def write_coord(self, path: str, full_precision: bool = True):
        """fg_write_coord: write_system's .coord of the current state."""
        self._check(lib().fg_write_coord(self._h, os.fsencode(path), 1 if full_precision else 0))

    # -- state
    def set_state(self, dipoR=None, dipoP=None, s=1.0, pi=0.0, H0=0.0):
        self._check(lib().fg_set_state(self._h, dptr(dipoR), dptr(dipoP), s, pi, H0))

    def set_thermostat(self, s, pi, H0):
        self._check(lib().fg_set_thermostat(self._h, s, pi, H0))

    def get_state(self) -> dict:
        u, q, f = real_field(self.p), real_field(self.p), real_field(self.p)
        strain = np.zeros(6)
        s, pi, H0 = C.c_double(), C.c_double(), C.c_double()
        self._check(lib().fg_get_state(self._h, dptr(u), dptr(q), dptr(f), dptr(strain),
                                       C.byref(s), C.byref(pi), C.byref(H0)))
        return dict(dipoR=u, dipoP=q, dVddi=f, strain=strain, s=s.value, pi=pi.value, H0=H0.value)

    def get_acouK(self) -> np.ndarray:
        a = complex_field(self.p)
        self._check(lib().fg_get_acouK(self._h, dptr(a.view(np.float64))))
        return a

    def set_uniform_E(self, E):
        e = np.ascontiguousarray(E, dtype=np.float64)
        self._check(lib().fg_set_uniform_E(self._h, dptr(e)))

    # -- hot path (reference subroutine names)
    def mirror_force_mirror(self, e: fg_energy | None = None) -> fg_energy:
        e = e if e is not None else fg_energy()
        self._check(lib().fg_mirror_force_mirror(self._h, C.byref(e)))
        return e

    def nose_poincare(self, e: fg_energy) -> fg_energy:
        self._check(lib().fg_nose_poincare(self._h, C.byref(e)))
        return e

    def leapfrog(self, e: fg_energy, i_step: int) -> fg_energy:
        self._check(lib().fg_leapfrog(self._h, C.byref(e), i_step))
        return e

    def upload_site_arrays(self, Z_starR=None, mass_dipo_inv=None, mass_acou_inv=None, relaxor=None, sum_p=None,
                           E_field_local=None):
        """fg_upload_site_arrays: padded Fortran-layout per-site arrays (int32
        for relaxor and sum_p); None keeps the default."""
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None
        dp_ = lambda a: dptr(a) if a is not None else None
        self._check(lib().fg_upload_site_arrays(self._h, dp_(Z_starR), dp_(mass_dipo_inv), dp_(mass_acou_inv),
                                                ip(relaxor), ip(sum_p), dp_(E_field_local)))

    def set_acou(self, acouR=None, acouP=None):
        """acouR / acouP (acoustic mass > 0), padded Fortran layout."""
        self._check(lib().fg_set_acou(self._h, dptr(acouR) if acouR is not None else None,
                                      dptr(acouP) if acouP is not None else None))

    def get_acou(self) -> dict:
        r, q, d = real_field(self.p), real_field(self.p), real_field(self.p)
        self._check(lib().fg_get_acou(self._h, dptr(r), dptr(q), dptr(d)))
        return {"acouR": r, "acouP": q, "dVdacR": d}

    def velocity_scaling(self, e: fg_energy) -> fg_energy:
        """velocity_scaling(p, c, e) of velocity_scaling.F:9-103."""
        self._check(lib().fg_velocity_scaling(self._h, C.byref(e)))
        return e

    def kinetic_energy_dipo(self) -> float:
        v = C.c_double()
        self._check(lib().fg_kinetic_energy_dipo(self._h, C.byref(v)))
        return v.value

    def nose_poincare_hamiltonian(self, e: fg_energy) -> fg_energy:
        self._check(lib().fg_nose_poincare_hamiltonian(self._h, C.byref(e)))
        return e

    def average_accumulate(self, e: fg_energy, avg: fg_average):
        self._check(lib().fg_average_accumulate(self._h, C.byref(e), C.byref(avg)))

    def run_steps(self, n: int, e: fg_energy | None = None) -> fg_energy:
        e = e if e is not None else fg_energy()
        self._check(lib().fg_run_steps(self._h, n, C.byref(e)))
        return e

    # -- sweep points and sample series
    def sample(self):
        """fg_sample: one row of the device sample series for this state."""
        self._check(lib().fg_sample(self._h))

    def samples(self) -> np.ndarray:
        """fg_samples_read: the rows held, (n, FG_SAMPLE_COLS); empties the series."""
        n = C.c_int()
        self._check(lib().fg_samples_read(self._h, None, 0, C.byref(n)))
        out = np.zeros((n.value, FG_SAMPLE_COLS))
        self._check(lib().fg_samples_read(self._h, dptr(out), n.value, C.byref(n)))
        return out

    def run_point(self, kelvin: float, n_therm: int, n_avg: int, every: int, E=None) -> fg_energy:
        """fg_run_point: chain to (kelvin, E), n_therm steps, n_avg steps with a
        sample row every `every` steps."""
        e = fg_energy()
        Ea = None if E is None else np.ascontiguousarray(E, dtype=np.float64)
        self._check(lib().fg_run_point(self._h, kelvin, dptr(Ea), n_therm, n_avg, every, C.byref(e)))
        p = fg_params()
        self._check(lib().fg_get_params(self._h, C.byref(p)))
        self.p = p
        return e

    # -- launch plans
    def tune(self, steps: int = 64):
        """fg_tune: time the plan candidates, keep the fastest; returns
        (z tile width, waves, ms per step)."""
        z, w, ms = C.c_int(), C.c_int(), C.c_double()
        self._check(lib().fg_tune(self._h, steps, C.byref(z), C.byref(w), C.byref(ms)))
        return z.value, w.value, ms.value

    def set_plan(self, zcw: int = 0, waves: int = 1):
        self._check(lib().fg_set_plan(self._h, zcw, waves))

    @property
    def plan(self):
        """(z tile width, waves, kick-drift grid, assembly grid)."""
        v = [C.c_int() for _ in range(4)]
        self._check(lib().fg_get_plan(self._h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def apply_wisdom(self):
        self._check(lib().fg_apply_wisdom(self._h))


class _Replica(Context):
    """A replica of a Batch: a Context view that the batch owns."""

    def __init__(self, handle, params, precision):  # noqa: super().__init__ would create a context
        self.p = params
        self.precision = precision
        self._h = C.c_void_p(handle)

    def close(self):
        self._h = C.c_void_p()


class Batch:
    """Independent replicas (sweep points of any sizes and methods) stepped
    together as one CUDA graph (fg_batch_create / fg_batch_step)."""

    def __init__(self, params_list, precision: int = FG_PREC_FP64):
        arr = (fg_params * len(params_list))(*params_list)
        self._b = C.c_void_p()
        eb = C.create_string_buffer(512)
        rc = lib().fg_batch_create(len(params_list), arr, precision, C.byref(self._b), eb, 512)
        if rc:
            raise FeramError(rc, _err(eb))
        self.replicas = [_Replica(lib().fg_batch_context(self._b, i), params_list[i], precision)
                         for i in range(len(params_list))]

    def __len__(self):
        return len(self.replicas)

    def __getitem__(self, i) -> Context:
        return self.replicas[i]

    def step(self, n_steps: int = 1):
        """n_steps steps of every replica; returns each replica's energies."""
        e = (fg_energy * len(self.replicas))()
        rc = lib().fg_batch_step(self._b, n_steps, e)
        if rc:
            r = lib().fg_batch_last_error(self._b)
            raise FeramError(rc, r.decode() if r else "")
        return list(e)

    def set_grouping(self, on: bool = True):
        """Replicas of one size step as one launch per kernel (default)."""
        lib().fg_batch_set_grouping(self._b, 1 if on else 0)

    def set_priorities(self, on: bool = True):
        """Branches of small supercells at a higher launch priority (default)."""
        lib().fg_batch_set_priorities(self._b, 1 if on else 0)

    @property
    def groups(self) -> int:
        """Branches of the last captured batch graph."""
        return lib().fg_batch_groups(self._b)

    def _bcheck(self, rc):
        if rc:
            r = lib().fg_batch_last_error(self._b)
            raise FeramError(rc, r.decode() if r else "")

    def run_point(self, kelvin, n_therm: int, n_avg: int, every: int, E=None):
        """fg_batch_run_point: every replica chained to its kelvin[i] (and
        E[i]), then n_therm + n_avg batch steps with sample rows."""
        k = np.ascontiguousarray(kelvin, dtype=np.float64)
        assert k.shape == (len(self.replicas),)
        Ea = None if E is None else np.ascontiguousarray(E, dtype=np.float64).reshape(len(self.replicas), 3)
        self._bcheck(lib().fg_batch_run_point(self._b, dptr(k), dptr(Ea), n_therm, n_avg, every))
        for r in self.replicas:
            p = fg_params()
            r._check(lib().fg_get_params(r._h, C.byref(p)))
            r.p = p

    def samples(self):
        """Every replica's sample series (emptied)."""
        return [r.samples() for r in self.replicas]

    def tune(self, steps: int = 16):
        """fg_batch_tune: per supercell, the fastest plan in whole batch steps;
        returns (ms per batch step before, after)."""
        a, b = C.c_double(), C.c_double()
        self._bcheck(lib().fg_batch_tune(self._b, steps, C.byref(a), C.byref(b)))
        return a.value, b.value

    def apply_wisdom(self):
        self._bcheck(lib().fg_batch_apply_wisdom(self._b))

    def close(self):
        if getattr(self, "_b", None):
            for r in self.replicas:
                r.close()
            lib().fg_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def wisdom_export() -> str:
    """fg_wisdom_export: the process's plans as text."""
    n = C.c_int()
    lib().fg_wisdom_export(None, 0, C.byref(n))
    buf = C.create_string_buffer(n.value)
    rc = lib().fg_wisdom_export(buf, n.value, C.byref(n))
    if rc:
        raise FeramError(rc, "fg_wisdom_export")
    return buf.value.decode()


def wisdom_import(text: str) -> int:
    """fg_wisdom_import: add the plans of `text`; returns how many."""
    n = C.c_int()
    rc = lib().fg_wisdom_import(text.encode(), C.byref(n))
    if rc:
        raise FeramError(rc, "malformed wisdom")
    return n.value


def wisdom_forget():
    lib().fg_wisdom_forget()


def wisdom_measure(p, n_times: int = 32, precision: int = FG_PREC_MIXED) -> str:
    """fg_wisdom_measure (feram_fftw_wisdom's role): tune the supercell of the
    run parameters p; returns the wisdom text afterwards."""
    eb = C.create_string_buffer(512)
    rc = lib().fg_wisdom_measure(C.byref(p), n_times, precision, eb, 512)
    if rc:
        raise FeramError(rc, _err(eb))
    return wisdom_export()


def feram_run(path: str, precision: int = FG_PREC_FP64):
    """feram_common + molecular_dynamics for one .feram file (writes .avg/.log)."""
    avg = fg_average()
    t = C.c_double()
    eb = C.create_string_buffer(512)
    rc = lib().fg_feram_run(os.fsencode(path), precision, C.byref(avg), C.byref(t), eb, 512)
    if rc:
        raise FeramError(rc, _err(eb))
    return avg, t.value
