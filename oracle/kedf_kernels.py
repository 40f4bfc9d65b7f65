"""Nonlocal KEDF kernels: Wang-Teter (LindG) and second-order WGC (ODE).

Restates ``LindG`` (Source/MathFunctions.f90:440-528), ``FillWT``
(Source/KEDF_WTkernel.f90:81-208) and the WGC kernel construction
(``FillWGC``/``FillWGC_ReciprocalSpace``, Source/KEDF_WGCkernel.f90:76-277, with
the ODE of ``makeKernel2``/``WGC``, Source/KEDF_KernelODE.f90:254-537).
Test infrastructure only.
"""
from __future__ import annotations

import functools
from fractions import Fraction

import numpy as np
from scipy.integrate import solve_ivp

from .cellsetup import spline_cubic_set, spline_cubic_val
from .consts import PI


def _lind_series_coefficients(nterms: int = 16):
    """Large-eta expansion of the inverse Lindhard function.

    With u = 1/eta^2, 1/2 + (1-eta^2)/(4 eta) ln|(1+eta)/(1-eta)| equals
    sum_{k>=1} u^k / ((2k-1)(2k+1)); inverting that series gives
    1/F = 3 eta^2 (1 + s1 u + s2 u^2 + ...).  Returns [3 s1, 3 s2, ...] as floats,
    the constant and the coefficients of u, u^2, ... in 1/F - 3 eta^2."""
    c = [Fraction(3, (2 * k - 1) * (2 * k + 1)) for k in range(1, nterms + 2)]  # c[0] = 1
    # S(u) = 1 / (1 + c1 u + c2 u^2 + ...), c_j = c[j]
    s = [Fraction(1)]
    for j in range(1, nterms + 1):
        acc = Fraction(0)
        for i in range(1, j + 1):
            acc += c[i] * s[j - i]
        s.append(-acc)
    return [float(3 * sj) for sj in s[1:]]


_LIND_SERIES = _lind_series_coefficients(16)  # constant term then 15 powers of u


def lind_g(eta, lam: float, mu: float):
    """Inverse Lindhard response minus TF and vW parts (MathFunctions.f90:440-528)."""
    eta = np.asarray(eta, float)
    out = np.empty_like(eta)
    neg = eta < 0.0
    small = (~neg) & (eta < 1e-10)
    one = (~neg) & (~small) & (np.abs(eta - 1.0) < 1e-10)
    big = (~neg) & (~small) & (~one) & (eta > 3.65)
    mid = ~(neg | small | one | big)
    out[neg] = 0.0
    e = eta[small]
    out[small] = 1.0 - lam + e ** 2 * (1.0 / 3.0 - 3.0 * mu)
    e = eta[one]
    out[one] = 2.0 - lam - 3.0 * mu + 20.0 * (e - 1.0)
    e = eta[big]
    e2 = e ** 2
    u = 1.0 / e2
    poly = np.zeros_like(e)
    for cf in reversed(_LIND_SERIES[1:]):
        poly = (poly + cf) * u
    out[big] = 3.0 * (1.0 - mu) * e2 - lam + _LIND_SERIES[0] + poly
    e = eta[mid]
    out[mid] = (1.0 / (0.5 + 0.25 * (1.0 - e ** 2) * np.log((1.0 + e) / np.abs(1.0 - e)) / e)
                - 3.0 * mu * e ** 2 - lam)
    return out


def wt_kernel(qtab: np.ndarray, rho0: float, alpha: float, beta: float, lam: float, mu: float) -> np.ndarray:
    """keKernel(:,:,:,1) = LindG(|G|/2kF) * 5 / (9 alpha beta rho0^(alpha+beta-5/3))
    (KEDF_WTkernel.f90:117-124,201)."""
    coef = 5.0 / (9.0 * alpha * beta * rho0 ** (alpha + beta - 5.0 / 3.0))
    tkf = 2.0 * (3.0 * rho0 * PI ** 2) ** (1.0 / 3.0)
    return lind_g(qtab / tkf, lam, mu) * coef


# ----------------------------------------------------------------------------
# WGC kernel
# ----------------------------------------------------------------------------
def wgc_eta_grid() -> np.ndarray:
    """The two-spacing eta grid of makeKernel2 (KEDF_KernelODE.f90:298-330)."""
    t_start1, t_end1, t_step1 = 1.0e-3, 3.0, 1.0e-3
    t_start2, t_end2, t_step2 = t_end1 + t_step1, 100.0, t_step1 * 10.0
    n1 = int(np.floor((t_end1 - t_start1) / t_step1)) - 1
    n2 = int(np.floor((t_end2 - t_start2) / t_step2)) - 1
    e1 = t_start1 + np.arange(n1, dtype=float) * t_step1
    e2 = t_start2 + np.arange(n2, dtype=float) * t_step2
    return np.concatenate([e1, e2])


def _wgc_rhs(beta: float, gamma: float):
    def rhs(t, y):
        eta = t
        if eta == 1.0:
            flind = 2.0
        elif eta == 0.0:
            flind = 1.0
        else:
            flind = 1.0 / (0.5 + (1.0 - eta ** 2) / (4.0 * eta) * np.log(abs((1.0 + eta) / (1.0 - eta))))
        yp2 = (20.0 * (flind - 3.0 * eta ** 2 - 1.0)
               - (gamma + 1.0 - 6.0 * 5.0 / 3.0) * eta * y[1]
               - 36.0 * (5.0 / 3.0 - beta) * beta * y[0]) / eta ** 2
        return np.array([y[1], yp2])
    return rhs


@functools.lru_cache(maxsize=8)
def wgc_radial_tables(alpha: float, beta: float, gamma: float, rtol: float = 1e-10):
    """Integrate the WGC kernel ODE inward from eta = 100 (KEDF_KernelODE.f90:254-478,481-537).

    Returns (eta, w, eta*w', eta^2*w''), matching what FillWGC_ReciprocalSpace
    splines (KEDF_WGCkernel.f90:166-176).  The reference integrates with RKSUITE
    RK(4,5) at TOL = 5e-5; this restatement uses a tighter LSODA integration
    (the equation is stiff near eta -> 0, where explicit Runge-Kutta steps shrink)."""
    eta = wgc_eta_grid()
    w_inf = -1.6 * 20.0 / (36.0 * alpha * beta)
    rhs = _wgc_rhs(beta, gamma)
    t_eval = eta[::-1]  # from eta(last) down to eta(1)
    sol = solve_ivp(rhs, (eta[-1], eta[0] * 0.9), [w_inf, 0.0], method="LSODA",
                    t_eval=t_eval, rtol=rtol, atol=1e-13)
    if not sol.success:
        raise RuntimeError("WGC kernel ODE failed: " + sol.message)
    y = sol.y[:, ::-1]
    w = y[0].copy()
    w1 = y[1].copy()
    w2 = np.array([rhs(t, y[:, i])[1] for i, t in enumerate(eta)])
    # the reference stores zeros at the starting point (KEDF_KernelODE.f90:351-353)
    w[-1] = 0.0
    w1[-1] = 0.0
    w2[-1] = 0.0
    return eta, w, eta * w1, eta ** 2 * w2


def wgc_kernels(qtab: np.ndarray, rho_s: float, gamma: float, tables) -> np.ndarray:
    """The four WGC kernel planes K0..K3 (KEDF_WGCkernel.f90:213-230)."""
    eta_t, w, w1, w2 = tables
    wpp = spline_cubic_set(eta_t, w, 0, 0.0, 0, 0.0)
    w1pp = spline_cubic_set(eta_t, w1, 0, 0.0, 0, 0.0)
    w2pp = spline_cubic_set(eta_t, w2, 0, 0.0, 0, 0.0)
    tkf_star = 2.0 * (3.0 * PI ** 2 * rho_s) ** (1.0 / 3.0)
    eta = (qtab / tkf_star).ravel()
    k1 = spline_cubic_val(eta_t, w, wpp, eta).reshape(qtab.shape)
    k2 = spline_cubic_val(eta_t, w1, w1pp, eta).reshape(qtab.shape)
    k3 = spline_cubic_val(eta_t, w2, w2pp, eta).reshape(qtab.shape)
    k4 = (k3 + (1.0 + gamma) * k2) / (36.0 * rho_s ** 2)
    k3 = (k3 + (7.0 - gamma) * k2) / (36.0 * rho_s ** 2)
    k2 = -k2 / (6.0 * rho_s)
    return np.stack([k1, k2, k3, k4])
