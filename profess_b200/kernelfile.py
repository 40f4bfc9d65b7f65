"""WT kernel files: the tabulated kernel the reference restarts from.

Format (FillWT_RestartFrom_GSpace, Source/KEDF_WTkernel.f90:212-408), text,
one value or pair per line: the KEDF type, the Fermi vector kF, the reference
density, the number of points nq, then nq lines "eta w(eta)" with eta = q/(2 kF)
ascending.  Reading multiplies w by the kernel prefactor and puts it on the
half spectrum by linear interpolation in eta = |q| / (2 kF) (the first value
below the table, an error above it); ``Engine.set_kernel`` then takes it.
"""
from __future__ import annotations

import numpy as np

WT_TYPE = 4  # the reference's kinetic code of Wang-Teter


def write_wt_kernel_file(path: str, kf: float, rho_s: float, eta: np.ndarray, w: np.ndarray) -> None:
    eta = np.asarray(eta, dtype=float)
    w = np.asarray(w, dtype=float)
    if eta.ndim != 1 or eta.shape != w.shape or np.any(np.diff(eta) <= 0):
        raise ValueError("eta must be a strictly increasing 1D table matching w")
    with open(path, "w") as fh:
        fh.write("%d\n%.17g\n%.17g\n%d\n" % (WT_TYPE, kf, rho_s, len(eta)))
        fh.writelines("%.17g %.17g\n" % (e, v) for e, v in zip(eta, w))


def read_wt_kernel_file(path: str):
    """(kedf type, kF, reference density, eta, w) as stored."""
    with open(path) as fh:
        tok = fh.read().split()
    kedf, kf, rho_s, nq = int(tok[0]), float(tok[1]), float(tok[2]), int(tok[3])
    vals = np.array(tok[4:4 + 2 * nq], dtype=float).reshape(nq, 2)
    return kedf, kf, rho_s, vals[:, 0].copy(), vals[:, 1].copy()


def wt_kernel_from_file(path: str, qnorm: np.ndarray, kf: float, coef: float) -> np.ndarray:
    """The kernel plane on the half spectrum (k1, n2, n3): coef * w(|q| / (2 kF))."""
    _, _, _, eta_in, w_in = read_wt_kernel_file(path)
    w_in = w_in * coef
    eta = np.asarray(qnorm, dtype=float) / (2.0 * kf)
    if eta.max() > eta_in[-1]:
        raise ValueError("the kernel file stops at eta = %g below the grid's %g" % (eta_in[-1], eta.max()))
    hi = np.clip(np.searchsorted(eta_in, eta, side="left"), 1, len(eta_in) - 1)
    lo = hi - 1
    d = eta_in[hi] - eta_in[lo]
    out = (eta_in[hi] - eta) / d * w_in[lo] + (eta - eta_in[lo]) / d * w_in[hi]
    return np.where(eta <= eta_in[0], w_in[0], out)
