"""Regenerate the committed golden fixtures of tests/golden from the reference tree.

Run where a checkout of the reference is available, giving its root:

    python tests/golden/make_golden.py <path to the reference checkout>

Every fixture is data the reference's own tests or examples hold:
  uni64_kat.json         marsaglia_tsang_uni64_check.F:11-16,22-40,42-46
  wave_kat.json          wave_check.f:8-35 (cases and parameters)
  modulation_kat.json    modulation_check.sh:8-79 (input deck, .modulation,
                         asserted log values and .coord vector)
  dispersion_long64.json doc/figures/BaTiO3-000-dispersion-with-ifc/
                         BaTiO3-000.dipole-dipole-long.dat + BaTiO3-000.param
  cooling16.json         src/03example-BaTiO3-bulk-phase-transition/
                         16x16x16-40000-10000/cooling.avg rows
  *.feram                src/zzznp.feram_check, zzz16.feram_check,
                         zzzlf.feram_check (parser fixtures)
The GPU box has no reference tree; tests read only these files.
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref: str):
    src = os.path.join(ref, "src")

    # uni64 known answers
    text = open(os.path.join(src, "marsaglia_tsang_uni64_check.F")).read()
    arr = re.search(r"r\(5\) = \(/(.*?)/\)", text, re.S).group(1)
    vals = [int(v) for v in re.findall(r"(\d{16})\.0d0", arr)]
    seeds = [int(x) for x in re.search(r"uni64\((\d+),(\d+)\)", text).groups()]
    ndraw = int(re.search(r"do i=1,(\d+)\s*\n\s*x=uni64\(\)", text).group(1))
    json.dump({"seed": seeds, "skip": ndraw, "next_times_2p53": vals}, open(os.path.join(HERE, "uni64_kat.json"), "w"),
              indent=1)

    # wave known answers: (type, i_step expression, expected expression)
    wt = open(os.path.join(src, "wave_check.f")).read()
    period = int(re.search(r"period\s*=\s*(\d+)", wt).group(1))
    n_th = int(re.search(r"n_thermalize\s*=\s*(\d+)", wt).group(1))
    amp = [float(a.replace("d0", "")) for a in re.search(r"amplitude\(3\)\s*=\s*\(/([^/]+)/\)", wt).group(1).split(",")]
    cases = []
    for m in re.finditer(r"x = wave\('(\w+)',\s*([^,]+),\s*n_thermalize, period, amplitude\); if \(x\((\d)\)\.ne\.\s*(.+?)\)\s+stop",
                         wt):
        kind, istep, comp, expect = m.group(1), m.group(2).strip(), int(m.group(3)), m.group(4).strip()
        env = {"period": period, "n_thermalize": n_th}
        istep_v = eval(istep, {}, env)
        ex = expect.replace("amplitude(1)", str(amp[0])).replace("amplitude(2)", str(amp[1])) \
                   .replace("amplitude(3)", str(amp[2])).replace("d0", "")
        cases.append({"type": kind, "i_step": istep_v, "comp": comp - 1, "expect": eval(ex)})
    json.dump({"period": period, "n_thermalize": n_th, "amplitude": amp, "cases": cases},
              open(os.path.join(HERE, "wave_kat.json"), "w"), indent=1)

    # modulation check
    sh = open(os.path.join(src, "modulation_check.sh")).read()
    deck = re.search(r"cat > zzzmodulation.feram <<-EOF\n(.*?)\nEOF", sh, re.S).group(1)
    deck = "\n".join(l.lstrip("\t") for l in deck.splitlines()) + "\n"
    mod = re.search(r"cat > zzzmodulation.modulation <<-EOF\n(.*?)\nEOF", sh, re.S).group(1)
    mod_pts = [[float(x) for x in l.split()] for l in mod.splitlines() if l.strip()]
    strain = re.search(r"inho_strain\s+\*(-?\d\\\.\d+)", sh).group(1).replace("\\", "")
    modv = re.search(r"inho_modulation \*(-?\d\\\.\d+)", sh).group(1).replace("\\", "")
    vec = re.search(r"' +(\d\\\.\d+E-\d+) '", sh).group(1).replace("\\", "")
    json.dump({"feram": deck, "modulation": mod_pts, "inho_strain_per_cell": strain,
               "inho_modulation_per_cell": modv, "acouR_abs": vec, "n_vectors_each_sign": 6,
               "n_log_lines": 3},
              open(os.path.join(HERE, "modulation_kat.json"), "w"), indent=1)

    # long-range dispersion
    d = os.path.join(ref, "doc", "figures", "BaTiO3-000-dispersion-with-ifc")
    par = {}
    for line in open(os.path.join(d, "BaTiO3-000.param")):
        k, v = line.split("=")
        par[k.strip()] = float(v)
    pts = []
    lines = open(os.path.join(d, "BaTiO3-000.dipole-dipole-long.dat")).read().splitlines()
    for i in range(0, len(lines), 4):
        f = lines[i].split()
        mat = [[float(x.replace("E", "e")) for x in lines[i + r].lstrip("#").split()] for r in (1, 2, 3)]
        pts.append({"k": [int(f[1]), int(f[2]), int(f[3])], "eig": [float(x.replace("E", "e")) for x in f[4:7]],
                    "matrix": mat})
    json.dump({"L": [int(par["Lx"]), int(par["Ly"]), int(par["Lz"])], "a0": par["a0"], "Z_star": par["Z_star"],
               "epsilon_inf": par["epsilon_inf"], "points": pts},
              open(os.path.join(HERE, "dispersion_long64.json"), "w"))

    # statistical golden: 16^3 cooling sweep (.avg rows)
    ex = os.path.join(src, "03example-BaTiO3-bulk-phase-transition", "16x16x16-40000-10000")
    rows = [[float(x) for x in l.split()] for l in open(os.path.join(ex, "cooling.avg")) if l.strip()]
    json.dump({"columns": "average_module.F:243-260", "n_thermalize": 40000, "n_average": 10000, "rows": rows},
              open(os.path.join(HERE, "cooling16.json"), "w"))

    # parser fixtures
    for name in ("zzznp.feram_check", "zzz16.feram_check", "zzzlf.feram_check"):
        txt = open(os.path.join(src, name)).read()
        open(os.path.join(HERE, name.replace(".feram_check", ".feram")), "w").write(txt)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path to the reference checkout>")
    main(sys.argv[1])
