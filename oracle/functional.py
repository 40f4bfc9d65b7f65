"""Energy/potential functional: ``CalculatePotentialPlus`` restated in FP64.

Follows Source/CalPotential.f90:41-647 for spin-unpolarised LDA with the
TF + vW + WT (kinetic = 4) or TF + vW + second-order WGC (kinetic = 5)
kinetic functionals.  The energy table has the reference layout
(Source/Report.f90:270-308): [total, KE, ion-e, Hartree, XC, ion-ion, TF, vW,
nonlocal], in Hartree.  Test infrastructure only.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .cellsetup import fft_c2r, fft_r2c
from .consts import C_TF, PI

KEDF_WT = 4
KEDF_WGC = 5


@dataclasses.dataclass
class Functional:
    """Module state that CalculatePotentialPlus reads through USE association."""
    kinetic: int            # 4 = WT, 5 = WGC
    n: tuple                # (n1, n2, n3)
    dv: float               # cell%dV
    qtab: np.ndarray        # |G| on the half spectrum (PlaneWave::qTable)
    kernel: np.ndarray      # (nplanes, k1, n2, n3) keKernel
    ion_pot: np.ndarray     # ionPotReal (n1, n2, n3)
    ion_ion: float          # Ewald::ionIonEnergy
    lam: float = 1.0
    mu: float = 1.0
    alpha: float = 5.0 / 6.0
    beta: float = 5.0 / 6.0
    rho_s: float = 0.0      # WGC expansion density rho*


# ---------------------------------------------------------------- LDA (PZ81)
def lda_energy_density_sum(rho: np.ndarray) -> float:
    """LDAEnergy for one spin channel (XC_LDA.f90:51-196)."""
    cX = -0.73855876638202234
    cC = 0.62035049089940009
    a, b, c, d = 3.11e-2, -4.8e-2, 2e-3, -1.16e-2
    g, b1, b2 = -1.423e-1, 1.0529, 3.334e-1
    exch = cX * np.sum(rho ** (4.0 / 3.0))
    rs = cC * rho ** (-1.0 / 3.0)
    lo = rs < 1
    ec = np.empty_like(rho)
    r = rs[lo]
    ec[lo] = np.log(r) * (a + c * r) + b + d * r
    r = rs[~lo]
    ec[~lo] = g / (1 + b1 * np.sqrt(r) + b2 * r)
    return float(exch + np.sum(rho * ec))


def lda_potential(rho: np.ndarray) -> np.ndarray:
    """LDAPot for one spin channel (XC_LDA.f90:199-310)."""
    cX = -0.98474502184269641
    cC = 0.62035049089940009
    cC1, cC2, cC3 = -5.83666666666666666e-2, 1.33333333333333333e-3, -8.4e-3
    cC4, cC5 = -0.174798948333333333, -6.325709333333333333e-2
    a1, g1, b1, b2 = 3.11e-2, -1.423e-1, 1.0529, 3.334e-1
    r13 = rho ** (1.0 / 3.0)
    rs = cC / r13
    out = np.empty_like(rho)
    lo = rs < 1
    r = rs[lo]
    out[lo] = cX * r13[lo] + np.log(r) * (a1 + cC2 * r) + cC1 + cC3 * r
    r = rs[~lo]
    sr = np.sqrt(r)
    out[~lo] = cX * r13[~lo] + (g1 + cC4 * sr + cC5 * r) / (1.0 + b1 * sr + b2 * r) ** 2
    return out


# ------------------------------------------------------------------ pieces
def hartree(f: Functional, rho: np.ndarray, q2: np.ndarray):
    """JPotentialPlus (Hartree.f90:93-169): V_H = IFFT(4 pi rho(G)/G^2), G=0 -> 0."""
    rg = fft_r2c(rho)
    with np.errstate(divide="ignore", invalid="ignore"):
        vg = np.where(q2 > 0.0, 4.0 * PI * rg / np.where(q2 > 0.0, q2, 1.0), 0.0)
    vg[0, 0, 0] = 0.0
    vh = fft_c2r(vg, f.n[0])
    return vh, float(np.sum(vh * rho) / 2.0)


def vw(f: Functional, sqrt_rho: np.ndarray, q2: np.ndarray):
    """VWPotentialSqrtPlus (KEDF_VW.f90:282-362): mu*IFFT(G^2 FFT(sqrt rho))."""
    lap = fft_c2r(fft_r2c(sqrt_rho) * q2, f.n[0])
    e = 0.5 * float(np.sum(sqrt_rho * lap)) * f.mu
    return lap * f.mu, e


def wt_potential(f: Functional, rho: np.ndarray):
    """WTPotPlus without the vacuum cutoff (KEDF_WT.f90:70-170)."""
    K = f.kernel[0]
    pb = fft_c2r(fft_r2c(rho ** f.beta) * K, f.n[0])
    e = C_TF * float(np.sum(rho ** f.alpha * pb))
    pa = fft_c2r(fft_r2c(rho ** f.alpha) * K, f.n[0])
    pot = C_TF * (f.alpha * rho ** (f.alpha - 1.0) * pb + f.beta * rho ** (f.beta - 1.0) * pa)
    return pot, e


def wgc_potential(f: Functional, rho: np.ndarray):
    """Second-order Taylor WGC, WGCT = 2, no vacuum cutoff (KEDF_WGC.f90:208-292)."""
    K1, K2, K3, K4 = f.kernel[0], f.kernel[1], f.kernel[2], f.kernel[3]
    n1 = f.n[0]
    a, b, rs = f.alpha, f.beta, f.rho_s
    theta = rho - rs
    rx = rho ** a
    Fr = fft_r2c(rx)
    Ft = fft_r2c(theta * rx)
    t0 = fft_r2c(theta * theta * rx / 2.0)
    work = fft_c2r(K1 * Fr + K2 * Ft + K3 * t0, n1)
    work2 = fft_c2r(K2 * Fr + K4 * Ft, n1)
    pot3 = fft_c2r(K3 * Fr, n1)
    rxb = rho ** b
    e = C_TF * float(np.sum(rxb * (work + theta * work2 + theta * theta / 2.0 * pot3)))
    pot = rho ** (b - 1.0) * (b * work + (rho + b * theta) * work2 + theta * (rho + b * theta / 2.0) * pot3)
    Fr = fft_r2c(rxb)
    Ft = fft_r2c(theta * rxb)
    t0 = fft_r2c(theta * theta * rxb / 2.0)
    work = fft_c2r(K1 * Fr + K2 * Ft + K3 * t0, n1)
    work2 = fft_c2r(K2 * Fr + K4 * Ft, n1)
    rxa = fft_c2r(K3 * Fr, n1)
    pot = pot + rho ** (a - 1.0) * (a * work + (rho + a * theta) * work2 + theta * (rho + a * theta / 2.0) * rxa)
    return pot * C_TF, e


def calculate_potential_plus(f: Functional, rho: np.ndarray, opt_sqrt: bool = True,
                             want_energy: bool = True):
    """CalculatePotentialPlus (CalPotential.f90:41-647) for numSpin = 1.

    Returns (potential, eTable or None).  With ``opt_sqrt`` the potential is
    dE/d(sqrt rho); otherwise dE/d rho."""
    loc = np.zeros(9)
    q2 = f.qtab ** 2
    pot = f.ion_pot.copy()                              # CalPotential.f90:200
    loc[2] = float(np.sum(rho * pot))                   # IonElectronEnergyReal
    vh, loc[3] = hartree(f, rho, q2)
    pot += vh
    pot += lda_potential(rho)
    if want_energy:
        loc[4] = lda_energy_density_sum(rho)
    # CalTF (KEDF_TF.f90:49-108)
    pot += (5.0 / 3.0 * C_TF * f.lam) * rho ** (2.0 / 3.0)
    loc[6] = f.lam * C_TF * float(np.sum(rho ** (5.0 / 3.0)))
    if f.kinetic == KEDF_WT:
        p9, loc[8] = wt_potential(f, rho)
    elif f.kinetic == KEDF_WGC:
        p9, loc[8] = wgc_potential(f, rho)
    else:
        raise ValueError("unsupported kinetic functional %r" % f.kinetic)
    pot += p9
    sq = np.sqrt(rho)
    if opt_sqrt:
        pot = 2.0 * sq * pot                            # CalPotential.f90:409-412
    lap, loc[7] = vw(f, sq, q2)
    if not opt_sqrt:
        lap = lap / (2.0 * sq)
    pot = pot + lap
    if not want_energy:
        return pot, None
    # CalculateEnergy (CalPotential.f90:610-644)
    loc[1] = loc[6:9].sum()
    et = loc * f.dv
    et[5] = f.ion_ion
    et[0] = et[1:6].sum()
    return pot, et
