"""Test infrastructure (the oracle): the stress tensor of a converged density,
a CPU restatement of CalculateStress (Source/CalStress.f90:44-253) for the WT
and the second-order WGC functionals with LDA, the B-spline ion-electron term
and the Ewald sum.  Only tests import it.  Stress = (1/volume) dE/d(strain),
Ha/bohr^3.

Terms:
  TF           -2/3 E_TF / vol on the diagonal            (TFStress, KEDF_TF.f90:283-334)
  vW           -mu <d_a sqrt(rho) d_b sqrt(rho)>          (VWStress, KEDF_VW.f90:365-449)
  WT           sum over the half spectrum of -eta G'(eta) F[rho^a] F[rho^b]* (q_a q_b / q^2
               - delta_ab / 3) pi^2 / (alpha beta kF rho0^(a+b-2)), - 2/3 E_WT / vol on the
               diagonal                                  (WTStress, KEDF_WT.f90:263-394)
  WGC          the kernel-derivative sums of WGCStress over the half spectrum of
               F[rho^x], x = a, b, a+1, b+1, a+2, b+2     (WGCStress, KEDF_WGC.f90:519-745)
  Hartree      8 pi sum_half |rho(q)|^2 q_a q_b / q^4 - E_H / vol   (JStress, Hartree.f90:173-247)
  LDA          E_xc / vol - <rho v_xc> on the diagonal   (LDAStress, XC_LDA.f90:663-732)
  ion-electron -2 N sum_half q_a q_b / q Re(rho(q) S_s(q)) V_s'(q), - E_ie, / vol
               (IonElectronStressSpline, IonElectronSpline.f90:359-534)
  Ewald        -(1/vol) dE_Ewald/d(strain), real and reciprocal sums and the
               neutralising-background term (EwaldStress, Ewald.f90:1857-2535), here from
               the strain derivatives of the oracle's own Ewald splitting
The half spectrum is qMask (PlaneWave.f90:255-296): the r2c half without the
kx = 0 (and Nyquist) plane's conjugate partners and self-conjugate points.
The tensor is symmetrised from its upper triangle, as the reference does.
"""
from __future__ import annotations

import math

import numpy as np

from . import cellsetup as cs
from . import functional as fn
from .consts import C_TF, PI


def q_mask(n1: int, n2: int, n3: int) -> np.ndarray:
    """qMask on the (k1, n2, n3) half spectrum, 1-based conditions of the serial branch."""
    k1, k2, k3 = n1 // 2 + 1, n2, n3
    offset = n1 % 2
    i1 = np.arange(1, k1 + 1)[:, None, None]
    i2 = np.arange(1, k2 + 1)[None, :, None]
    i3 = np.arange(1, k3 + 1)[None, None, :]
    half2 = (i2 >= 2) & (i2 <= (k2 - 1) // 2 + 1)
    half3 = (i3 >= 2) & (i3 <= (k3 - 1) // 2 + 1)
    plane = (half2 | ((i2 == 1) & half3) | ((k2 % 2 == 0) & (i2 == k2 // 2 + 1) & half3))
    m = ((offset == 1) & (i1 >= 2)) | ((offset == 0) & (i1 >= 2) & (i1 < k1))
    m = m | ((i1 == 1) & plane) | ((offset == 0) & (i1 == k1) & plane)
    return np.broadcast_to(m, (k1, k2, k3)).copy()


def g_prime(eta: np.ndarray, mu: float) -> np.ndarray:
    """Derivative of the Lindhard-based WT function (GPrime, MathFunctions.f90:531-578)."""
    eta = np.asarray(eta, float)
    out = np.zeros_like(eta)
    small = (eta >= 0) & (eta < 1e-10)
    one = np.abs(eta - 1.0) < 1e-10
    gen = (eta >= 1e-10) & ~one
    e = eta[gen]
    out[small] = 2.0 * eta[small] * (1.0 / 3.0 - 3.0 * mu)
    out[one] = 40.0
    out[gen] = (((e ** 2 + 1.0) * 0.25 / e ** 2 * np.log(np.abs((1.0 + e) / (1.0 - e))) - 0.5 / e)
                / (0.5 + 0.25 * (1.0 - e ** 2) * np.log((1.0 + e) / np.abs(1.0 - e)) / e) ** 2 - 6.0 * e * mu)
    return out


def psp_diff_lookup(sp: cs.Species, q: np.ndarray) -> np.ndarray:
    """dV/dq by the same index-knot spline (PseudoPotDiffLookup, LocalPseudoPot.f90:207-276)."""
    q = np.asarray(q, float)
    n = len(sp.pot_values)
    dq = sp.max_g / float(n - 1)
    out = np.zeros_like(q)
    ok = (q <= sp.max_g) & (q > 0)
    pos = q[ok] / dq + 1.0
    left = np.clip(np.floor(pos).astype(np.int64), 1, n - 1)
    dt = pos - left
    yl, yr = sp.vqs[left - 1], sp.vqs[left]
    pl, pr = sp.pot_dd[left - 1], sp.pot_dd[left]
    # derivative of the cubic on unit knot spacing (spline_cubic_val's ypval)
    yp = (yr - yl) - (pr / 6.0 + pl / 3.0) + dt * (pl + dt * 0.5 * (pr - pl))
    out[ok] = yp / dq + 8.0 * PI * float(sp.charge) / q[ok] ** 3
    return out


def _outer(g, w):
    """sum over points of w * g_a g_b, as a 3x3 array."""
    g = np.asarray(g).reshape(-1, 3)
    return np.einsum("na,nb,n->ab", g, g, np.asarray(w).reshape(-1))


def ewald_stress(lattice: np.ndarray, frac: np.ndarray, z: np.ndarray) -> np.ndarray:
    vol = abs(np.linalg.det(lattice))
    recip = np.linalg.inv(lattice).T * 2.0 * PI
    pos = frac @ lattice.T
    nion = len(z)
    eta = math.sqrt(PI) * (max(nion, 1) / vol ** 2) ** (1.0 / 6.0)
    rcut, gcut = 7.0 / eta, 2.0 * eta * 7.0
    inv = np.linalg.inv(lattice)
    nimg = [int(math.ceil(rcut * np.linalg.norm(inv[a]))) + 1 for a in range(3)]
    ng = [int(math.ceil(gcut * np.linalg.norm(lattice[:, a]) / (2 * PI))) + 1 for a in range(3)]
    s = np.zeros((3, 3))
    e_real = 0.0
    for a in range(-nimg[0], nimg[0] + 1):
        for b in range(-nimg[1], nimg[1] + 1):
            for c in range(-nimg[2], nimg[2] + 1):
                t = lattice @ np.array([a, b, c], float)
                d = pos[None, :, :] + t[None, None, :] - pos[:, None, :]
                r2 = (d * d).sum(axis=2)
                ok = (r2 > 1e-24) & (r2 < rcut * rcut)
                r = np.sqrt(r2[ok])
                zz = (z[:, None] * z[None, :])[ok]
                dv = d[ok]
                ec = np.array([math.erfc(eta * x) for x in r]) / r
                e_real += 0.5 * float((zz * ec).sum())
                fp = -ec / r - 2.0 * eta / math.sqrt(PI) * np.exp(-eta * eta * r * r) / r   # f'(r)
                s += 0.5 * _outer(dv, zz * fp / r)
    m = np.stack(np.meshgrid(*[np.arange(-k, k + 1) for k in ng], indexing="ij"), -1).reshape(-1, 3)
    m = m[np.any(m != 0, axis=1)]
    G = m @ recip.T
    g2 = (G * G).sum(axis=1)
    keep = g2 <= gcut * gcut
    G, g2, m = G[keep], g2[keep], m[keep]
    ph = 2.0 * PI * (m @ frac.T)
    sf2 = (z[None, :] * np.cos(ph)).sum(1) ** 2 + (z[None, :] * np.sin(ph)).sum(1) ** 2
    fg = np.exp(-g2 / (4 * eta * eta)) / g2
    e_rec = 2 * PI / vol * float((fg * sf2).sum())
    s += 2 * PI / vol * _outer(G, fg * sf2 * 2.0 * (1.0 / (4 * eta * eta) + 1.0 / g2))
    e_bg = -0.5 * PI / (eta * eta) / vol * float(z.sum()) ** 2
    s -= np.eye(3) * (e_rec + e_bg)
    return s / vol


def wgc_stress(cell: cs.Cell, f: fn.Functional, rho: np.ndarray, gamma: float, rho0: float) -> np.ndarray:
    """WGCStress (Source/KEDF_WGC.f90:519-745) for the second-order WGC kernel
    (WGCT = 2) with rho0 and rho* not held (hold0 = holdS = .FALSE.): upper
    triangle, before CalculateStress symmetrises."""
    n1, n2, n3 = f.n
    g = cs.g_vectors(cell.recip, n1, n2, n3)
    q = np.sqrt((g * g).sum(-1))
    mask = q_mask(n1, n2, n3)
    qm = np.where(mask, q, 1.0)
    a, b, rs, mu = f.alpha, f.beta, f.rho_s, f.mu
    kf = (3.0 * PI ** 2 * rs) ** (1.0 / 3.0)
    fa = np.conj(cs.fft_r2c(rho ** a))
    fb = cs.fft_r2c(rho ** b)
    fa1 = np.conj(cs.fft_r2c(rho ** (a + 1.0)))
    fb1 = cs.fft_r2c(rho ** (b + 1.0))
    fa2 = np.conj(cs.fft_r2c(rho ** (a + 2.0)))
    fb2 = cs.fft_r2c(rho ** (b + 2.0))
    ki = 20.0 * rho0 ** (5.0 / 3.0 - (a + b))
    c001, c002, c003 = -2.0 / 3.0, rs * 4.0 / 3.0, -rs ** 2 * 2.0 / 3.0
    c011, c012, c021, c111 = -5.0 / 3.0, rs * 5.0 / 3.0, -4.0 / 3.0, -8.0 / 3.0
    c011, c012, c021, c111, diff = c011 + 1.0, c012 - rs, c021 + 1.0, c111 + 2.0, -1.0 / 3.0
    K1, K2, K3, K4 = f.kernel[0], f.kernel[1], f.kernel[2], f.kernel[3]
    eta = np.where(mask, q / (2.0 * kf), 0.0)
    c00 = c001 * K1 + c002 * K2 + c003 * (K3 + K4)
    c01 = c011 * K2 + c012 * (K3 + K4)
    c02 = c021 * K3
    c11 = c111 * K4
    diago = fa * c00 * fb + fa1 * c01 * fb + fa * c01 * fb1 + fa2 * c02 * fb + fa * c02 * fb2 + fa1 * c11 * fb1
    gp = g_prime(eta, mu)
    d11 = -ki * eta / (36.0 * rs ** 2) * gp - K4 * 6.0 * (a + b) - K2 * (gamma * (a + b) + 6.0 * a * b) / rs
    d02 = (-ki * eta / (72.0 * rs ** 2) * gp - K4 * (3.0 * (a + b + 1.0) - gamma)
           - K2 * (3.0 * gamma * (a + b + 1.0) - gamma ** 2 + 18.0 * a * b) / (6.0 * rs))
    d01 = K4 * 6.0 * rs + K2 * gamma
    d00 = 6.0 * rs * K2 - 2.0 * rs * d01 + rs ** 2 * (2.0 * d02 + d11)
    d01 = -rs * (d11 + 2.0 * d02) + d01
    offdia = fa * d00 * fb + fa1 * d01 * fb + fa * d01 * fb1 + fa2 * d02 * fb + fa * d02 * fb2 + fa1 * d11 * fb1
    dg = float(np.where(mask, np.real(diago + offdia * diff), 0.0).sum())
    s = np.eye(3) * dg + _outer(g, np.where(mask, np.real(offdia) / qm ** 2, 0.0))
    return np.triu(s) * 2.0 * C_TF


def stress(cell: cs.Cell, f: fn.Functional, rho: np.ndarray, gamma: float = 2.7, rho0: float = None) -> np.ndarray:
    """The stress tensor (Ha/bohr^3) of density rho for the WT or WGC functional
    f (gamma and rho0: the WGC kernel's parameters; rho0 defaults to N / V)."""
    assert f.kinetic in (fn.KEDF_WT, fn.KEDF_WGC)
    n1, n2, n3 = f.n
    N = n1 * n2 * n3
    vol = cell.vol
    _, et = fn.calculate_potential_plus(f, rho)
    g = cs.g_vectors(cell.recip, n1, n2, n3)
    q = np.sqrt((g * g).sum(-1))
    mask = q_mask(n1, n2, n3)
    qm = np.where(mask, q, 1.0)
    s = np.zeros((3, 3))
    eye = np.eye(3)
    # TF
    s += -2.0 / 3.0 * et[6] / vol * eye
    # vW: real-space mean of the gradient products of sqrt(rho)
    sq = cs.fft_r2c(np.sqrt(rho))
    grads = [cs.fft_c2r(1j * g[..., a] * sq, n1) for a in range(3)]
    for a in range(3):
        for b in range(a, 3):
            s[a, b] += -f.mu * float((grads[a] * grads[b]).sum()) / N
    if f.kinetic == fn.KEDF_WGC:
        s += wgc_stress(cell, f, rho, gamma, cell.num_electrons / vol if rho0 is None else rho0)
    else:  # WT
        rho0 = cell.num_electrons / vol
        kf = (3.0 * PI ** 2 * rho0) ** (1.0 / 3.0)
        fa = cs.fft_r2c(rho ** f.alpha)
        fb = np.conj(cs.fft_r2c(rho ** f.beta))
        eta = np.where(mask, q / (2.0 * kf), 0.0)
        diff = np.where(mask, np.real(-eta * g_prime(eta, f.mu) * fa * fb), 0.0)
        wt = _outer(g, diff / qm ** 2) - eye / 3.0 * float(diff.sum())
        s += wt * PI ** 2 / (f.alpha * f.beta * kf * rho0 ** (f.alpha + f.beta - 2.0))
        s += -2.0 / 3.0 * et[8] / vol * eye
    # Hartree
    rq = cs.fft_r2c(rho)
    s += 8.0 * PI * _outer(g, np.where(mask, np.abs(rq) ** 2 / qm ** 4, 0.0)) - et[3] / vol * eye
    # LDA
    s += (et[4] / vol - float((rho * fn.lda_potential(rho)).sum()) / N) * eye
    # ion-electron, B-spline structure factor
    b1 = cs.bspline_b(cs.SPLINE_ORDER, n1 // 2 + 1, n1)
    b2 = cs.bspline_b(cs.SPLINE_ORDER, n2, n2)
    b3 = cs.bspline_b(cs.SPLINE_ORDER, n3, n3)
    ie = np.zeros((3, 3))
    for sidx, sp in enumerate(cell.species):
        sel = cell.species_of_ion == sidx
        if not np.any(sel):
            continue
        sfac = cs.fft_r2c(cs.fill_q_ion_table(cell.frac[sel], cs.SPLINE_ORDER, n1, n2, n3))
        sfac = sfac * b1[:, None, None] * b2[None, :, None] * b3[None, None, :]
        vp = psp_diff_lookup(sp, qm.ravel()).reshape(q.shape)
        w = np.where(mask, np.real(rq * sfac) * vp / qm, 0.0)
        ie += _outer(g, w)
    s += (-2.0 * N * ie - et[2] * eye) / vol
    # Ewald
    s += ewald_stress(cell.lattice, cell.frac, cell.charges())
    # symmetrise from the upper triangle
    return np.triu(s) + np.triu(s, 1).T
