"""Test infrastructure (the oracle): FillWT_RestartFrom_GSpace's interpolation
(Source/KEDF_WTkernel.f90:212-408) with its own bisection, point by point.
Only tests import it."""
from __future__ import annotations

import numpy as np


def wt_kernel_loops(eta_in, w_in, qnorm, kf: float, coef: float) -> np.ndarray:
    w_in = np.asarray(w_in, float) * coef
    nq = len(eta_in)
    out = np.zeros(qnorm.shape)
    for idx in np.ndindex(qnorm.shape):
        eta = qnorm[idx] / (2.0 * kf)
        if eta <= eta_in[0]:
            out[idx] = w_in[0]
        elif eta > eta_in[nq - 1]:
            out[idx] = w_in[nq - 1]
        else:
            i1, i2 = 0, nq - 1
            while i1 < i2 - 1:
                mid = (i1 + i2) // 2
                if eta > eta_in[mid]:
                    i1 = mid
                else:
                    i2 = mid
            f1 = (eta_in[i2] - eta) / (eta_in[i2] - eta_in[i1])
            f2 = (eta - eta_in[i1]) / (eta_in[i2] - eta_in[i1])
            out[idx] = f1 * w_in[i1] + f2 * w_in[i2]
    return out
