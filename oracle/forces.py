"""Post-solve ion forces: Ewald plus the B-spline ion-electron term.

Restates ``ForcesII_IE`` (Source/CalForce.f90:134-239),
``IonElectronForcesSpline`` (Source/IonElectronSpline.f90:219-355) and
``CalculateSplineForces`` (Source/IonElectronSpline.f90:642-753).
Test infrastructure only.
"""
from __future__ import annotations

import numpy as np

from .cellsetup import (SPLINE_ORDER, Cell, bspline_b, cardinal_bspline, fft_c2r,
                        fft_r2c, psp_lookup, q_table)
from .ewald import ewald


def ion_electron_forces_spline(cell: Cell, rho: np.ndarray, order: int = SPLINE_ORDER) -> np.ndarray:
    n1, n2, n3 = rho.shape
    k1 = n1 // 2 + 1
    rho_g = fft_r2c(rho)
    qn = q_table(cell.recip, n1, n2, n3)
    b1 = bspline_b(order, k1, n1)
    b2 = bspline_b(order, n2, n2)
    b3 = bspline_b(order, n3, n3)
    bprod = b1[:, None, None] * b2[None, :, None] * b3[None, None, :]
    cell_inv = np.linalg.inv(cell.lattice).T
    out = np.zeros((len(cell.frac), 3))
    for s, sp in enumerate(cell.species):
        sel = np.nonzero(cell.species_of_ion == s)[0]
        if len(sel) == 0:
            continue
        psp = psp_lookup(sp, qn.ravel()).reshape(qn.shape)
        psp[0, 0, 0] = 0.0
        factor = fft_c2r(rho_g * psp * bprod, n1)
        for i in sel:
            gc = cell.frac[i] * np.array([n1, n2, n3], dtype=float)
            fl = np.floor(gc)
            x = gc - fl
            M = [cardinal_bspline(order, x[d]) for d in range(3)]
            # order-1 splines in an array of length order+1, last entry zero (CBSpline.f90:56)
            D = [np.append(cardinal_bspline(order - 1, x[d]), 0.0) for d in range(3)]
            idx = np.arange(order)
            l1 = np.mod(int(fl[0]) - idx, n1)
            l2 = np.mod(int(fl[1]) - idx, n2)
            l3 = np.mod(int(fl[2]) - idx, n3)
            m1, m2, m3 = M[0][1:order + 1], M[1][1:order + 1], M[2][1:order + 1]
            d1 = (D[0][1:order + 1] - D[0][0:order]) * n1
            d2 = (D[1][1:order + 1] - D[1][0:order]) * n2
            d3 = (D[2][1:order + 1] - D[2][0:order]) * n3
            fac = factor[l1[:, None, None], l2[None, :, None], l3[None, None, :]]
            q1 = (d1[:, None, None] * m2[None, :, None] * m3[None, None, :] * fac).sum()
            q2 = (m1[:, None, None] * d2[None, :, None] * m3[None, None, :] * fac).sum()
            q3 = (m1[:, None, None] * m2[None, :, None] * d3[None, None, :] * fac).sum()
            out[i] = -(cell_inv @ np.array([q1, q2, q3]))
    return out


def total_forces(cell: Cell, rho: np.ndarray):
    """Returns (total, ewald, ion-electron) forces in Ha/bohr, each (nion, 3)."""
    _, f_ii = ewald(cell.lattice, cell.frac, cell.charges(), want_forces=True)
    f_ie = ion_electron_forces_spline(cell, rho)
    return f_ii + f_ie, f_ii, f_ie
