"""Density files: the reference's ``.den`` format, written and read on the host.

Layout (PrintDensity / Print3DArray, Source/Output.f90:617-953; ReadDensity,
Source/ReadIonFile.f90:1054-1314): fixed 27-character records.  Records 1-4
are a 14-character label and a 12-character integer (x, y and z dimension,
number of spins); then one value per record in Fortran E26.20 form, x fastest,
then y, then z, then spin.  The reference writes them as formatted direct-access
records; this module ends each record with a newline and reads records that
end in a newline or a blank.

Reading onto a grid of another size interpolates trilinearly between the
file's points (periodic), with the reference's cell-centred mapping
frac = (L_file * repeat / L_grid * (1 + 2 i) - 1) / 2; a grid that is exactly
``repeat`` times the file's copies it.  Either way the density is then scaled
to hold the cell's electrons.
"""
from __future__ import annotations

import math

import numpy as np

RECL = 27
_LABELS = ("x-dimension:", "y-dimension:", "z-dimension:", "# of spins: ")


# Smallest magnitude the two-digit exponent of E26.20 holds (.1E-98); smaller
# values are written as zero so that every record keeps RECL characters.
_E26_MIN = 1.0e-99


def _e26_20(x: float) -> str:
    """x in Fortran E26.20 form: sign, '.', 20 digits, 'E', sign, 2 digits (no leading 0).

    Values below 1e-99 in magnitude (a vacuum region's density) are written as
    zero; a non-finite value or one of 1e99 or more raises ValueError, since
    either would break the fixed record length."""
    if not math.isfinite(x):
        raise ValueError("non-finite density value %r cannot be written in E26.20" % x)
    if abs(x) < _E26_MIN:
        return " .00000000000000000000E+00"
    s = "%.19e" % abs(x)                  # d.dddddddddddddddddddde[+-]XX
    mant, ex = s.split("e")
    digits = mant.replace(".", "")
    e = int(ex) + 1
    if abs(e) > 99:
        raise ValueError("density value %r is outside the E26.20 exponent range" % x)
    body = ".%sE%s%02d" % (digits, "-" if e < 0 else "+", abs(e))
    return ("-" if x < 0 else " ") + body


def write_density(path: str, rho: np.ndarray) -> None:
    """Write one spin density (n1, n2, n3), x fastest (PrintDensity without the
    size cap's down-sampling)."""
    rho = np.asarray(rho, dtype=np.float64)
    n1, n2, n3 = rho.shape
    with open(path, "w") as fh:
        for lab, v in zip(_LABELS, (n1, n2, n3, 1)):
            fh.write("%-14s%12d\n" % (lab, v))
        flat = rho.ravel(order="F")
        fh.write("".join(_e26_20(float(v)) + "\n" for v in flat))


def _records(path: str):
    with open(path, "rb") as fh:
        data = fh.read()
    nrec = len(data) // RECL
    return [data[k * RECL:(k + 1) * RECL] for k in range(nrec)]


def read_density_file(path: str) -> np.ndarray:
    """The file's density as stored, shape (nx, ny, nz, nspin)."""
    recs = _records(path)
    dims = [int(r[14:26]) for r in recs[:4]]
    nx, ny, nz, ns = dims
    vals = np.array([float(r[:26]) for r in recs[4:4 + nx * ny * nz * ns]], dtype=np.float64)
    return vals.reshape((nx, ny, nz, ns), order="F")


def _axis_map(n_grid: int, n_file: int, repeat: int):
    """Per grid index: lower file index, upper file index (periodic) and weight."""
    i = np.arange(n_grid, dtype=np.float64)
    frac = (float(n_file * repeat) / float(n_grid) * (1.0 + 2.0 * i) - 1.0) * 0.5
    frac = np.mod(frac, float(n_file))
    lo = frac.astype(np.int64)
    w = frac - lo
    hi = np.where(lo == n_file - 1, 0, lo + 1)
    return lo, hi, w


def read_density(path: str, grid, num_electrons: float, volume: float, repeat=(1, 1, 1)) -> np.ndarray:
    """ReadDensity for one spin: the file's density on ``grid`` (copied when the
    grid is the file's times ``repeat``, interpolated otherwise), scaled so that
    it integrates to ``num_electrons`` over ``volume``."""
    f = read_density_file(path)
    if f.shape[3] != 1:
        raise ValueError("the file holds %d spin densities; one is expected" % f.shape[3])
    f = f[..., 0]
    n = tuple(int(x) for x in grid)
    if all(f.shape[a] * repeat[a] == n[a] for a in range(3)):
        rho = np.tile(f, repeat)
    else:
        (x0, x1, wx), (y0, y1, wy), (z0, z1, wz) = (_axis_map(n[a], f.shape[a], repeat[a]) for a in range(3))
        wx, wy, wz = wx[:, None, None], wy[None, :, None], wz[None, None, :]

        def plane(z):
            a = f[x0][:, y0][:, :, z] * (1 - wx) + f[x1][:, y0][:, :, z] * wx
            b = f[x0][:, y1][:, :, z] * (1 - wx) + f[x1][:, y1][:, :, z] * wx
            return a * (1 - wy) + b * wy

        rho = plane(z0) * (1 - wz) + plane(z1) * wz
    total = float(rho.sum())
    scale = float(num_electrons) * math.prod(n) / (total * float(volume))
    return np.asfortranarray(rho * scale)
