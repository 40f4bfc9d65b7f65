"""Local pseudopotential tables in the CASTEP .recpot format.

Reading follows ``ReadPseudo`` (Source/ReadIonFile.f90:821-976): values in
eV*A^3 on a uniform q grid up to maxG (A^-1) are converted to Ha*bohr^3 and
bohr^-1, the ionic charge is inferred from the -4 pi Z / q^2 tail of the first
two points, and V(q) + 4 pi Z / q^2 is splined over the point index with zero
end slopes.  The engine evaluates that spline on the device
(``ofdft_slot_build_ion_potential``).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

BOHR = 0.529177208607388                     # Source/Constants.f90:56
_QE, _C = 1.602176462e-19, 299792458.0
_EPS0 = 1.0 / (4.0 * math.pi * 1e-7 * _C ** 2)
HARTREE_TO_EV = _QE * 1e10 / (4.0 * math.pi * _EPS0 * BOHR)   # Source/Constants.f90:74


@dataclasses.dataclass
class Species:
    name: str
    charge: int
    max_g: float            # bohr^-1
    pot_values: np.ndarray  # Ha*bohr^3
    vqs: np.ndarray
    pot_dd: np.ndarray


def _spline_second_derivatives_unit(y: np.ndarray, yp0: float, ypn: float) -> np.ndarray:
    """spline_cubic_set with knots 1..n (unit spacing) and given end slopes
    (ibcbeg = ibcend = 1), by the Thomas algorithm."""
    n = len(y)
    sub = np.full(n, 1.0 / 6.0)
    diag = np.full(n, 2.0 / 3.0)
    sup = np.full(n, 1.0 / 6.0)
    r = np.empty(n)
    r[1:-1] = (y[2:] - y[1:-1]) - (y[1:-1] - y[:-2])
    r[0] = (y[1] - y[0]) - yp0
    diag[0], sup[0] = 1.0 / 3.0, 1.0 / 6.0
    r[-1] = ypn - (y[-1] - y[-2])
    sub[-1], diag[-1] = 1.0 / 6.0, 1.0 / 3.0
    cp = np.empty(n)
    dp = np.empty(n)
    cp[0] = sup[0] / diag[0]
    dp[0] = r[0] / diag[0]
    for i in range(1, n):
        m = diag[i] - sub[i] * cp[i - 1]
        cp[i] = sup[i] / m if i < n - 1 else 0.0
        dp[i] = (r[i] - sub[i] * dp[i - 1]) / m
    x = np.empty(n)
    x[-1] = dp[-1]
    for i in range(n - 2, -1, -1):
        x[i] = dp[i] - cp[i] * x[i + 1]
    return x


def species_from_table(max_g_ang: float, values_ev_a3, name: str = "X") -> Species:
    vals = np.array(values_ev_a3, dtype=float)
    if vals[-1] == 1000.0:
        vals[-1] = 0.0
    vals = vals / (BOHR ** 3 * HARTREE_TO_EV)
    max_g = max_g_ang * BOHR
    n = len(vals)
    dq = max_g / float(n - 1)
    charge = int(np.rint(-(vals[1] - vals[0]) * dq ** 2 / (4.0 * math.pi)))
    t = np.arange(1, n + 1, dtype=float)
    vqs = vals.copy()
    vqs[1:] = vals[1:] + 4.0 * math.pi * charge / (((t[1:] - 1.0) / float(n - 1) * max_g) ** 2)
    return Species(name, charge, max_g, vals, vqs, _spline_second_derivatives_unit(vqs, 0.0, 0.0))


def parse_recpot(text: str, name: str = "X") -> Species:
    lines = text.splitlines()
    k = next(i for i, ln in enumerate(lines) if "END COMMENT" in ln)
    max_g_ang = float(lines[k + 2].split()[0])
    records = [ln for ln in lines[k + 3:] if ln.strip()]
    if not records or records[-1].split()[0] != "1000":
        raise ValueError("Pseudopotential lacks the proper terminator")
    npts = 3 * len(records) - 3
    toks = []
    for ln in records:
        toks.extend(ln.split())
    return species_from_table(max_g_ang, [float(x) for x in toks[:npts]], name)


def format_recpot(max_g_ang: float, values_ev_a3, comment: str = "") -> str:
    """Write a table in the layout ReadPseudo reads (three values per line, 1000 terminator)."""
    out = ["START COMMENT", "  " + comment, "END COMMENT", "3     5", "     %.16f" % max_g_ang]
    v = list(values_ev_a3)
    for i in range(0, len(v), 3):
        out.append("  ".join("%.16E" % x for x in v[i:i + 3]))
    out.append("  1000")
    return "\n".join(out) + "\n"
