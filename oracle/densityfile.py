"""Test infrastructure (the oracle): ReadDensity's interpolation
(Source/ReadIonFile.f90:1054-1314) restated with explicit loops, one spin.
Only tests import it."""
from __future__ import annotations

import math

import numpy as np


def read_density_loops(f: np.ndarray, grid, num_electrons: float, volume: float, repeat=(1, 1, 1)) -> np.ndarray:
    """f: the file's values (xLen, yLen, zLen) -> the density on ``grid``."""
    xl, yl, zl = f.shape
    nx, ny, nz = grid
    rho = np.zeros(grid)
    if xl * repeat[0] == nx and yl * repeat[1] == ny and zl * repeat[2] == nz:
        for iz in range(nz):
            for iy in range(ny):
                for ix in range(nx):
                    rho[ix, iy, iz] = f[ix % xl, iy % yl, iz % zl]
    else:
        def split(i, n, length, rep):
            fr = (float(length * rep) / float(n) * (1.0 + 2.0 * i) - 1.0) * 0.5
            fr = fr % float(length)
            ind = int(fr)
            return ind, fr - ind, (length if ind == length - 1 else 0)

        for iz in range(nz):
            iz0, dz, sz = split(iz, nz, zl, repeat[2])
            for iy in range(ny):
                iy0, dy, sy = split(iy, ny, yl, repeat[1])
                for ix in range(nx):
                    ix0, dx, sx = split(ix, nx, xl, repeat[0])

                    def plane(kz):
                        d1 = f[ix0, iy0, kz]
                        d2 = f[ix0 + 1 - sx, iy0, kz]
                        d3 = f[ix0, iy0 + 1 - sy, kz]
                        d4 = f[ix0 + 1 - sx, iy0 + 1 - sy, kz]
                        return (d1 * (1 - dx) + d2 * dx) * (1 - dy) + (d3 * (1 - dx) + d4 * dx) * dy

                    rho[ix, iy, iz] = plane(iz0) * (1 - dz) + plane(iz0 + 1 - sz) * dz
    return rho * (num_electrons * math.prod(grid) / (rho.sum() * volume))
