"""Shared inputs of the tests: parameter decks, seeded configurations,
error measures."""
import json
import os
import re

import numpy as np

from feram_b200 import _capi as A

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    path = os.path.join(GOLDEN, name)
    if name.endswith(".json"):
        return json.load(open(path))
    return open(path).read()


def deck(base="zzznp.feram", **tags):
    """A reference input deck with some tags replaced or added.

    Values are written verbatim (strings must carry their quotes)."""
    text = golden(base)
    for k, v in tags.items():
        line = f"{k} = {v}"
        pat = re.compile(rf"^\s*{re.escape(k)}\s*=.*$", re.M)
        if pat.search(text):
            text = pat.sub(line, text)
        else:
            text += "\n" + line + "\n"
    return text


def params(base="zzznp.feram", **tags):
    import feram_b200
    return feram_b200.params_from_text(deck(base, **tags), "t")


def seeded_u(p, seed, sigma=0.1, avg=0.0):
    """u ~ N(avg, sigma) per component from uni64 seed (seed, 987654321),
    in the reference's draw order (initialize-dipoR.F:41-54)."""
    import ctypes as C
    q = A.fg_params.from_buffer_copy(p)
    q.seed[0], q.seed[1] = seed, 987654321
    for a in range(3):
        q.init_dipo_avg[a] = avg
        q.init_dipo_dev[a] = sigma
        q.k_stripe[a] = 0.0
    u = A.real_field(p)
    rc = A.lib().fg_init_dipoR_host(C.byref(q), A.dptr(u), None)
    assert rc == 0
    return u


def fp32_config(u):
    """The configuration rounded to FP32: the state the mixed path holds
    (its fields are FP32).  Parity of the mixed path is measured on such
    configurations, given identically to the FP64 oracle; the effect of the
    rounding itself is a property of FP32 state, reported apart."""
    return u.astype(np.float32).astype(np.float64)


def seeded_p(p, seed, sigma=0.02):
    return seeded_u(p, seed + 5000, sigma=sigma)


def force_error(F, Fref, p):
    """(max, rms) over sites of |F - Fref| / rms |Fref| (physical sites)."""
    d = A.physical(F, p) - A.physical(Fref, p)
    ref = A.physical(Fref, p)
    rms = np.sqrt(np.mean(np.sum(ref ** 2, axis=-1)))
    n = np.sqrt(np.sum(d ** 2, axis=-1))
    return float(n.max() / rms), float(np.sqrt(np.mean(n ** 2)) / rms)


def energy_errors(e, eref, fields=A.POTENTIAL_FIELDS):
    """Per-term |dE| / max(|E_ref|, 1e-3 * sum |E_ref terms|)."""
    scale = sum(abs(getattr(eref, f)) for f in fields)
    out = {}
    for f in fields:
        r = getattr(eref, f)
        out[f] = abs(getattr(e, f) - r) / max(abs(r), 1e-3 * scale, 1e-300)
    return out
