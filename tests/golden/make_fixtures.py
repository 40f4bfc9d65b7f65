"""Generate the golden fixtures from the reference's own test runs.

Reads the input geometries, the Al pseudopotential table and the printed
energy/trajectory tables of the reference's shipped sample outputs (its
``test`` directory) and writes them as small fixtures next to this file:

  ref_cases.json     geometries, KEDF parameters and golden numbers (with the
                     source file:line of every number)
  al_hc_recpot.npz   the al_HC.lda.recpot table (maxG in 1/A, values in eV*A^3)

The fixtures are committed so that tests never need the reference tree.
Run:  python tests/golden/make_fixtures.py REFERENCE_ROOT
(or set PROFESS_REFERENCE to the root of the reference's source tree).
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

REF = None  # the reference's test directory, set by main()
HERE = os.path.dirname(os.path.abspath(__file__))


def _lines(path):
    with open(path) as fh:
        return fh.read().splitlines()


def _ion_block(path):
    text = open(path).read()

    def block(name):
        m = re.search(r"%BLOCK\s+" + name + r"(.*?)%END\s*BLOCK\s+" + name, text, re.S | re.I)
        return [ln.split() for ln in m.group(1).strip().splitlines() if ln.strip()]

    lat = [[float(x) for x in r[:3]] for r in block("LATTICE_CART")]
    pos = [[r[0]] + [float(x) for x in r[1:4]] for r in block("POSITIONS_FRAC")]
    return {"lattice_angstrom_rows": lat, "positions_frac": pos}


def _find(lines, pattern, rel):
    for i, ln in enumerate(lines):
        m = re.search(pattern, ln)
        if m:
            return float(m.group(1).replace("D", "E")), "%s:%d" % (rel, i + 1)
    raise ValueError("pattern not found: " + pattern)


def _trajectory(lines, rel):
    rows = []
    for i, ln in enumerate(lines):
        m = re.match(r"\|\s+(\d+)\s+(-?\d\.\d+E[+-]\d+)\s+(\d\.\d+E[+-]\d+)\s+(\d+)/\s*(\d+)\s+(\d\.\d+E[+-]\d+)", ln)
        if m:
            rows.append({"step": int(m.group(1)), "energy_ev": float(m.group(2)),
                         "pot_norm": float(m.group(3)), "ncg": int(m.group(4)),
                         "nline": int(m.group(5)), "theta": float(m.group(6)),
                         "source": "%s:%d" % (rel, i + 1)})
            if len(rows) > 1 and rows[-1]["step"] == 0:
                rows.pop()
                break
    return rows


def _stress_au(lines, rel):
    """The first STRESS (a.u.) block: rows 'ST_AU  i  s_i1 s_i2 s_i3' (Ha/bohr^3)."""
    rows, src = [], []
    for i, ln in enumerate(lines):
        m = re.match(r"\s*ST_AU\s+(\d)\s+(\S+)\s+(\S+)\s+(\S+)", ln)
        if m:
            rows.append([float(m.group(k).replace("D", "E")) for k in (2, 3, 4)])
            src.append(i + 1)
            if len(rows) == 3:
                break
    return {"value": rows, "source": "%s:%d-%d" % (rel, src[0], src[-1])}


def _cell_relax(lines, rel, geom_path, geom_rel):
    """The cell relaxation trace: per cell step the TOTAL ENERGY (eV) of its
    density solve, the ST_AU stress (Ha/bohr^3) and the step's summary line;
    then the final lattice (Angstrom rows) of the .final.geom file."""
    steps, energy, stress, src = [], None, [], None
    for i, ln in enumerate(lines):
        m = re.search(r"TOTAL ENERGY =\s+(\S+) eV", ln)
        if m:
            energy, src = float(m.group(1)), i + 1
        m = re.match(r"\s*ST_AU\s+(\d)\s+(\S+)\s+(\S+)\s+(\S+)", ln)
        if m:
            stress.append([float(m.group(k).replace("D", "E")) for k in (2, 3, 4)])
        m = re.search(r"; Cell optimization at step\s*(\d+), max\(stress\):\s*(\S+), total energy:\s*(\S+)", ln)
        if m:
            steps.append({"step": int(m.group(1)), "energy_ev": energy, "energy_source": "%s:%d" % (rel, src),
                          "stress_au": stress[-3:], "max_stress": float(m.group(2)),
                          "energy_ha_line": float(m.group(3)), "source": "%s:%d" % (rel, i + 1)})
            stress = []
    final = _ion_block(geom_path)
    return {"steps": steps, "final_lattice_angstrom_rows": final["lattice_angstrom_rows"],
            "final_source": geom_rel, "max_cell_step": 100, "tols": 5.0e-7,
            "params_source": "Source/CellOptimizers.f90 (maxCellStep, tols)"}


def _final_terms(lines, rel, nonlocal_label):
    labels = {"tf": r"Thomas-Fermi Kin\. Energy =\s+(\S+) eV",
              "vw": r"Von-Weizsacker Kin\. Ener =\s+(\S+) eV",
              "nonlocal": nonlocal_label + r"\s+=\s+(\S+) eV",
              "xc": r"LDA Exch-Corr Energy =\s+(\S+) eV",
              "hartree": r"Coulombic Energy =\s+(\S+) eV",
              "ion_electron": r"Ion-Electron Energy =\s+(\S+) eV",
              "ion_ion": r"Ion-Ion Energy =\s+(\S+) eV",
              "total": r"TOTAL ENERGY =\s+(\S+) eV"}
    out = {}
    for k, pat in labels.items():
        v, src = _find(lines, pat, rel)
        out[k] = {"value_ev": v, "source": src}
    return out


def main(root=None):
    global REF
    root = root or os.environ.get("PROFESS_REFERENCE")
    if not root:
        raise SystemExit("usage: make_fixtures.py REFERENCE_ROOT (or set PROFESS_REFERENCE)")
    REF = os.path.join(root, "test")
    cases = {}
    # WT: displaced Al4 (first density solve of the ion relaxation)
    rel = "test/optIon/sampleoutput/displaced.out"
    lines = _lines(os.path.join(REF, "optIon/sampleoutput/displaced.out"))
    traj = _trajectory(lines, rel)
    fmax, fsrc = _find(lines, r"max_force=\s+(\S+)", rel)
    cases["wt_al4_displaced"] = {
        "geometry": _ion_block(os.path.join(REF, "optIon/displaced.ion")),
        "geometry_source": "test/optIon/displaced.ion",
        "ecut_ev": 600.0, "kinetic": "WT", "lambda": 1.0, "mu": 1.0,
        "alpha": 5.0 / 6.0, "beta": 5.0 / 6.0,
        "grid": [16, 16, 16], "grid_source": rel + ":19",
        "dv": _find(lines, r"dV of each real space grid is now\s+(\S+)", rel),
        "trajectory": traj,
        "final": _final_terms(lines, rel, r"Wang-Teter Kinetic Energ"),
        "max_force_ha_bohr": {"value": fmax, "source": fsrc},
    }
    # WGC: ideal FCC Al4
    rel = "test/optDen/sample.output"
    lines = _lines(os.path.join(REF, "optDen/sample.output"))
    cases["wgc_al4_fcc"] = {
        "geometry": _ion_block(os.path.join(REF, "optDen/Al4.ion")),
        "geometry_source": "test/optDen/Al4.ion",
        "ecut_ev": 600.0, "kinetic": "WGC", "lambda": 1.0, "mu": 1.0,
        "alpha": 1.2060113295832982827348622781219,
        "beta": 0.46065533708336838393180438854479,
        "gamma": 2.7, "params_source": "test/optDen/test.inpt:5-6",
        "grid": [16, 16, 16], "grid_source": rel + ":19",
        "dv": _find(lines, r"dV of each real space grid is now\s+(\S+)", rel),
        "fermi_vector": _find(lines, r"Fermi vector :\s+(\S+)", rel),
        "reference_density": _find(lines, r"Reference density :\s+(\S+)", rel),
        "trajectory": _trajectory(lines, rel),
        "final": _final_terms(lines, rel, r"WGC Kinetic Energy"),
    }
    # WT: optCell first solve (undisplaced ions in the sheared cell)
    rel = "test/optCell/sampleoutput/displaced.out"
    lines = _lines(os.path.join(REF, "optCell/sampleoutput/displaced.out"))
    cases["wt_al4_cell"] = {
        "geometry": _ion_block(os.path.join(REF, "optCell/displaced.ion")),
        "geometry_source": "test/optCell/displaced.ion",
        "ecut_ev": 600.0, "kinetic": "WT", "lambda": 1.0, "mu": 1.0,
        "alpha": 5.0 / 6.0, "beta": 5.0 / 6.0,
        "trajectory": _trajectory(lines, rel),
        "final": {"total": dict(zip(("value_ev", "source"),
                                    _find(lines, r"TOTAL ENERGY =\s+(\S+) eV", rel)))},
        "stress_au": _stress_au(lines, rel),
        "cell_relax": _cell_relax(lines, rel, os.path.join(REF, "optCell/sampleoutput/displaced.final.geom"),
                                  "test/optCell/sampleoutput/displaced.final.geom"),
    }
    for c in cases.values():
        c["dv"] = dict(zip(("value", "source"), c["dv"])) if "dv" in c else None
        for k in ("fermi_vector", "reference_density"):
            if k in c:
                c[k] = dict(zip(("value", "source"), c[k]))
    with open(os.path.join(HERE, "ref_cases.json"), "w") as fh:
        json.dump(cases, fh, indent=1)

    # the Al local pseudopotential table shared by all three runs
    rp = _lines(os.path.join(REF, "optIon/al_HC.lda.recpot"))
    k = next(i for i, ln in enumerate(rp) if "END COMMENT" in ln)
    max_g = float(rp[k + 2].split()[0])
    toks = []
    for ln in rp[k + 3:]:
        toks.extend(ln.split())
    assert toks[-1] == "1000"
    vals = np.array([float(t) for t in toks[:-1]])
    np.savez_compressed(os.path.join(HERE, "al_hc_recpot.npz"), max_g=max_g, values=vals,
                        source="test/optIon/al_HC.lda.recpot")
    print("wrote", len(cases), "cases;", len(vals), "recpot values")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
