"""Ion-ion Ewald energy and forces (restates the sums of Source/Ewald.f90).

The reference evaluates E_ion-ion = real-space sum + self term + reciprocal sum
+ average-potential (neutralising background) term (Ewald.f90:465-520,
1150-1190).  This restatement evaluates the same four terms with the exact
reciprocal sum (the reference's default uses a B-spline/PME reciprocal part,
Ewald.f90:993-1147) converged to ~1e-13 Ha, with its own splitting parameter.
Test infrastructure only.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erfc

from .consts import PI


def _images(lattice: np.ndarray, rcut: float) -> np.ndarray:
    inv = np.linalg.inv(lattice)
    # number of images along each axis so that every point within rcut is covered
    heights = 1.0 / np.sqrt((inv ** 2).sum(axis=1))
    n = [int(math.ceil(rcut / h)) + 1 for h in heights]
    r = [np.arange(-k, k + 1) for k in n]
    I, J, K = np.meshgrid(*r, indexing="ij")
    m = np.stack([I.ravel(), J.ravel(), K.ravel()], axis=1).astype(float)
    return m @ lattice.T  # (nimg, 3) cartesian translations


def _recip_points(recip: np.ndarray, gcut: float) -> np.ndarray:
    inv = np.linalg.inv(recip)
    heights = 1.0 / np.sqrt((inv ** 2).sum(axis=1))
    n = [int(math.ceil(gcut / h)) + 1 for h in heights]
    r = [np.arange(-k, k + 1) for k in n]
    I, J, K = np.meshgrid(*r, indexing="ij")
    m = np.stack([I.ravel(), J.ravel(), K.ravel()], axis=1).astype(float)
    g = m @ recip.T
    g2 = (g ** 2).sum(axis=1)
    keep = (g2 > 0.0) & (g2 <= gcut * gcut)
    return g[keep]


def ewald(lattice: np.ndarray, frac: np.ndarray, charges: np.ndarray, want_forces: bool = False):
    """Return (energy in Ha, forces (nion,3) in Ha/bohr or None)."""
    vol = abs(np.linalg.det(lattice))
    recip = np.linalg.inv(lattice).T * 2.0 * PI
    pos = frac @ lattice.T
    nion = len(charges)
    eta = math.sqrt(PI) * (max(nion, 1) / vol ** 2) ** (1.0 / 6.0)
    rcut = 7.0 / eta
    gcut = 2.0 * eta * 7.0
    # real space
    trans = _images(lattice, rcut)
    e_real = 0.0
    f = np.zeros((nion, 3))
    for i in range(nion):
        d = pos[None, :, :] + trans[:, None, :] - pos[i][None, None, :]  # (img, j, 3)
        r = np.sqrt((d ** 2).sum(axis=-1))
        mask = (r > 1e-12) & (r < rcut)
        rr = np.where(mask, r, 1.0)
        term = np.where(mask, erfc(eta * rr) / rr, 0.0)
        e_real += 0.5 * charges[i] * (term * charges[None, :]).sum()
        if want_forces:
            dterm = np.where(mask, -erfc(eta * rr) / rr ** 2
                             - 2.0 * eta / math.sqrt(PI) * np.exp(-(eta * rr) ** 2) / rr, 0.0)
            # dE/dR_i = -sum_j Z_i Z_j dterm * d/r  (d = R_j + L - R_i)
            g = (dterm * charges[None, :])[..., None] * d / rr[..., None]
            f[i] += charges[i] * g.sum(axis=(0, 1))
    e_self = -eta / math.sqrt(PI) * float((charges ** 2).sum())
    gv = _recip_points(recip, gcut)
    g2 = (gv ** 2).sum(axis=1)
    phase = gv @ pos.T                      # (ng, nion)
    s = (charges[None, :] * np.exp(1j * phase)).sum(axis=1)
    fg = np.exp(-g2 / (4.0 * eta * eta)) / g2
    e_rec = 2.0 * PI / vol * float((fg * np.abs(s) ** 2).sum())
    e_bg = -0.5 * PI / eta ** 2 / vol * float(charges.sum()) ** 2
    energy = e_real + e_self + e_rec + e_bg
    if not want_forces:
        return energy, None
    im = np.imag(np.conj(s)[:, None] * np.exp(1j * phase))  # (ng, nion)
    f_rec = 4.0 * PI / vol * charges[:, None] * ((fg[:, None] * im)[..., None] * gv[:, None, :]).sum(axis=0)
    return energy, f + f_rec
