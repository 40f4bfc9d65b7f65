"""Cell, grid, plane-wave and ion-potential setup (FP64 restatement).

Restates the host-side setup of PROFESS that feeds the density solve:
geometry and pseudopotential reading, FFT grid sizing, the |G| table, the
cubic-spline local pseudopotential lookup, and the Choly-Kaxiras cardinal
B-spline ion-electron potential.  Test infrastructure only (see package doc).
"""
from __future__ import annotations

import dataclasses
import math
import re

import numpy as np
import scipy.fft as sfft
from scipy.linalg import solve_banded

from .consts import BOHR, HARTREE_TO_EV, PI

SPLINE_ORDER = 10  # Source/CBSpline.f90:36


# ----------------------------------------------------------------------------
# FFT convention of the reference (Source/Fourier_v1.f90:333-465)
# ----------------------------------------------------------------------------
# Threads of the oracle's FFTs (scipy.fft workers): -1 = every host core; a
# timing of the oracle on one core sets 1.
FFT_WORKERS = -1


def fft_r2c(a: np.ndarray) -> np.ndarray:
    """Forward 3D real->half-complex FFT scaled by 1/N (Fourier_v1.f90:389-393).

    ``a`` has shape (n1, n2, n3); the result has shape (n1//2+1, n2, n3)."""
    return sfft.rfftn(a, axes=(1, 2, 0), norm="forward", workers=FFT_WORKERS)


def fft_c2r(c: np.ndarray, n1: int) -> np.ndarray:
    """Backward 3D half-complex->real FFT, unscaled (Fourier_v1.f90:400-465)."""
    _, n2, n3 = c.shape
    return sfft.irfftn(c, s=(n2, n3, n1), axes=(1, 2, 0), norm="forward", workers=FFT_WORKERS)


# ----------------------------------------------------------------------------
# Geometry and pseudopotentials
# ----------------------------------------------------------------------------
@dataclasses.dataclass
class Species:
    name: str
    charge: int            # ionic charge inferred from the recpot tail
    max_g: float           # bohr^-1
    pot_values: np.ndarray  # V(q) in Ha*bohr^3 on the uniform q grid
    vqs: np.ndarray        # V(q) + 4 pi Z / q^2 (spline knots)
    pot_dd: np.ndarray     # spline second derivatives


@dataclasses.dataclass
class Cell:
    lattice: np.ndarray    # (3,3) bohr; column i is lattice vector i
    frac: np.ndarray       # (nion, 3) fractional coordinates
    species_of_ion: np.ndarray  # (nion,) index into species
    species: list

    @property
    def vol(self) -> float:
        return float(abs(np.linalg.det(self.lattice)))

    @property
    def recip(self) -> np.ndarray:
        """cellRecip = TRANSPOSE(Inverse(cellReal)) * 2 pi (CellInfo.f90:281)."""
        return np.linalg.inv(self.lattice).T * 2.0 * PI

    @property
    def lengths(self) -> np.ndarray:
        return np.sqrt((self.lattice ** 2).sum(axis=0))

    @property
    def num_electrons(self) -> int:
        return int(sum(self.species[s].charge for s in self.species_of_ion))

    def charges(self) -> np.ndarray:
        return np.array([self.species[s].charge for s in self.species_of_ion], dtype=float)


def parse_recpot_text(text: str, name: str = "X") -> Species:
    """Read a CASTEP .recpot table the way ReadPseudo does (ReadIonFile.f90:821-976).

    The number of points is 3 * (records after the maxG line) - 3; the record
    count includes the closing "1000" line (ReadIonFile.f90:856-863)."""
    lines = text.splitlines()
    k = next(i for i, ln in enumerate(lines) if "END COMMENT" in ln)
    # line k+1 is the "3 5" version line; line k+2 is maxG; then the data
    max_g_ang = float(lines[k + 2].split()[0])
    records = [ln for ln in lines[k + 3:] if ln.strip() != ""]
    if not records or records[-1].split()[0] != "1000":
        raise ValueError("Pseudopotential lacks the proper terminator")
    num_points = 3 * len(records) - 3
    toks = []
    for ln in records:
        toks.extend(ln.split())
    vals = np.array([float(t) for t in toks[:num_points]], dtype=float)
    if len(vals) < num_points:
        raise ValueError("recpot data shorter than declared")
    return species_from_table(max_g_ang, vals, name)


def species_from_table(max_g_ang: float, values_ev_a3: np.ndarray, name: str = "X") -> Species:
    """Species from a recpot table: maxG in A^-1 and V(q) in eV*A^3.

    Converts to Ha*bohr^3 and bohr^-1, infers the ionic charge from the first
    two points and sets up the cubic spline of V(q) + 4 pi Z / q^2 over the
    point index with zero end slopes (ReadIonFile.f90:914-976)."""
    vals = np.array(values_ev_a3, dtype=float)
    if vals[-1] == 1000.0:  # ReadIonFile.f90:914-917
        vals[-1] = 0.0
    vals = vals / (BOHR ** 3 * HARTREE_TO_EV)
    max_g = max_g_ang * BOHR
    num_points = len(vals)
    dq = max_g / float(num_points - 1)
    charge = int(np.rint(-(vals[1] - vals[0]) * dq ** 2 / (4.0 * PI)))
    t = np.arange(1, num_points + 1, dtype=float)
    vqs = vals.copy()
    vqs[1:] = vals[1:] + 4.0 * PI * charge / (((t[1:] - 1.0) / float(num_points - 1) * max_g) ** 2)
    pot_dd = spline_cubic_set(t, vqs, 1, 0.0, 1, 0.0)
    return Species(name=name, charge=charge, max_g=max_g, pot_values=vals, vqs=vqs, pot_dd=pot_dd)


def spline_cubic_set(t, y, ibcbeg, ybcbeg, ibcend, ybcend) -> np.ndarray:
    """Second derivatives of the interpolating cubic spline (MathSplines.f90:178-393).

    Boundary flags: 0 = quadratic end interval, 1 = given slope, 2 = given
    second derivative."""
    t = np.asarray(t, float)
    y = np.asarray(y, float)
    n = len(t)
    rhs = np.zeros(n)
    sub = np.zeros(n)   # sub[i] multiplies ypp[i-1]
    diag = np.zeros(n)
    sup = np.zeros(n)   # sup[i] multiplies ypp[i+1]
    if ibcbeg == 0:
        rhs[0], diag[0], sup[0] = 0.0, 1.0, -1.0
    elif ibcbeg == 1:
        rhs[0] = (y[1] - y[0]) / (t[1] - t[0]) - ybcbeg
        diag[0] = (t[1] - t[0]) / 3.0
        sup[0] = (t[1] - t[0]) / 6.0
    else:
        rhs[0], diag[0], sup[0] = ybcbeg, 1.0, 0.0
    i = np.arange(1, n - 1)
    rhs[i] = (y[i + 1] - y[i]) / (t[i + 1] - t[i]) - (y[i] - y[i - 1]) / (t[i] - t[i - 1])
    sub[i] = (t[i] - t[i - 1]) / 6.0
    diag[i] = (t[i + 1] - t[i - 1]) / 3.0
    sup[i] = (t[i + 1] - t[i]) / 6.0
    if ibcend == 0:
        rhs[n - 1], sub[n - 1], diag[n - 1] = 0.0, -1.0, 1.0
    elif ibcend == 1:
        rhs[n - 1] = ybcend - (y[n - 1] - y[n - 2]) / (t[n - 1] - t[n - 2])
        sub[n - 1] = (t[n - 1] - t[n - 2]) / 6.0
        diag[n - 1] = (t[n - 1] - t[n - 2]) / 3.0
    else:
        rhs[n - 1], sub[n - 1], diag[n - 1] = ybcend, 0.0, 1.0
    ab = np.zeros((3, n))
    ab[0, 1:] = sup[:-1]
    ab[1, :] = diag
    ab[2, :-1] = sub[1:]
    return solve_banded((1, 1), ab, rhs)


def spline_cubic_val(t, y, ypp, tval):
    """Evaluate the spline at ``tval`` (MathSplines.f90:395-496); vectorised.

    Out-of-range arguments use the first or last interval, as rvec_bracket does."""
    t = np.asarray(t, float)
    tval = np.asarray(tval, float)
    left = np.searchsorted(t, tval, side="right") - 1
    left = np.clip(left, 0, len(t) - 2)
    right = left + 1
    dt = tval - t[left]
    h = t[right] - t[left]
    tmp1 = (y[right] - y[left]) / h
    tmp2 = -(ypp[right] / 6.0 + ypp[left] / 3.0) * h
    tmp3 = ypp[right] - ypp[left]
    return y[left] + dt * (tmp1 + tmp2 + dt * (0.5 * ypp[left] + dt * (tmp3 / (6.0 * h))))


def psp_lookup(sp: Species, q: np.ndarray) -> np.ndarray:
    """V_loc(|q|) by the index-knot cubic spline (LocalPseudoPot.f90:92-202)."""
    q = np.asarray(q, float)
    out = np.zeros_like(q)
    n = len(sp.pot_values)
    dq = sp.max_g / float(n - 1)
    zero = q == 0.0
    big = q >= sp.max_g
    mid = ~(zero | big)
    qm = q[mid]
    pos = qm / dq + 1.0
    left = np.floor(pos).astype(np.int64)      # 1-based
    dt = pos - left
    yl = sp.vqs[left - 1]
    yr = sp.vqs[left]
    pl = sp.pot_dd[left - 1]
    pr = sp.pot_dd[left]
    yval = yl + dt * (yr - yl - (pr / 6.0 + pl / 3.0) + dt * (0.5 * pl + dt * ((pr - pl) / 6.0)))
    out[mid] = yval - 4.0 * PI * float(sp.charge) / qm ** 2
    out[zero] = sp.pot_values[0]
    return out


def parse_ion_file(text: str, recpots: dict) -> Cell:
    """Minimal reader for the reference's .ion blocks (ReadIonFile.f90).

    Supports LATTICE_CART (Angstrom, one lattice vector per line),
    POSITIONS_FRAC and SPECIES_POT; ``recpots`` maps species name to recpot text or a Species."""
    def block(name):
        m = re.search(r"%BLOCK\s+" + name + r"(.*?)%END\s*BLOCK\s+" + name, text, re.S | re.I)
        if not m:
            raise ValueError("missing block " + name)
        return [ln.split() for ln in m.group(1).strip().splitlines() if ln.strip()]

    lat_rows = block("LATTICE_CART")
    lat = np.array([[float(x) for x in r[:3]] for r in lat_rows])  # row i = vector i
    lattice = lat.T / BOHR  # column i = vector i (Fortran READ fills columns)
    pos = block("POSITIONS_FRAC")
    sp_rows = block("SPECIES_POT")
    names = [r[0] for r in sp_rows]
    species = [recpots[nm] if isinstance(recpots[nm], Species) else parse_recpot_text(recpots[nm], nm)
               for nm in names]
    idx = np.array([names.index(r[0]) for r in pos], dtype=np.int64)
    frac = np.array([[float(x) for x in r[1:4]] for r in pos])
    return Cell(lattice=lattice, frac=frac, species_of_ion=idx, species=species)


# ----------------------------------------------------------------------------
# Grid sizing (SetupFFT.f90:193-382, dimType = 1)
# ----------------------------------------------------------------------------
def pad_fft_dim(r: float) -> int:
    """Smallest 2^a 3^b 5^c 7^d >= r (PadFFTdims, SetupFFT.f90:300-380)."""
    eps = 1.0e-14
    log_r = math.log(r)
    p2 = int(log_r / math.log(2.0) - eps + 1)
    p3 = int(log_r / math.log(3.0) - eps + 1)
    p5 = int(log_r / math.log(5.0) - eps + 1)
    p7 = int(log_r / math.log(7.0) - eps + 1)
    minimum = 7 ** p7
    for i7 in range(p7 + 1):
        for i5 in range(p5 + 1):
            for i3 in range(p3 + 1):
                for i2 in range(0, p2 + 1):
                    tr = 7 ** i7 * 5 ** i5 * 3 ** i3 * 2 ** i2
                    if tr >= r:
                        if tr < minimum:
                            minimum = tr
                        break
    return minimum


def size_system(ecut_ha: float, lattice: np.ndarray) -> tuple:
    """Grid dims from the cutoff: m = sqrt(2 Ecut) * |a_i| / pi (SetupFFT.f90:237-247)."""
    q_max = math.sqrt(ecut_ha * 2.0)
    lengths = np.sqrt((lattice ** 2).sum(axis=0))
    return tuple(pad_fft_dim(q_max * L / PI) for L in lengths)


def g_vectors(recip: np.ndarray, n1: int, n2: int, n3: int) -> np.ndarray:
    """G vectors on the half spectrum (FillQTable, PlaneWave.f90:215-236).

    m1 = i1 (no wrap); m2, m3 wrap above n/2, so the Nyquist index stays +n/2."""
    k1 = n1 // 2 + 1
    m1 = np.arange(k1, dtype=float)
    m2 = np.arange(n2, dtype=float)
    m2[m2 > n2 // 2] -= n2
    m3 = np.arange(n3, dtype=float)
    m3[m3 > n3 // 2] -= n3
    M1, M2, M3 = np.meshgrid(m1, m2, m3, indexing="ij")
    g = (recip[:, 0][None, None, None, :] * M1[..., None]
         + recip[:, 1][None, None, None, :] * M2[..., None]
         + recip[:, 2][None, None, None, :] * M3[..., None])
    return g


def q_table(recip: np.ndarray, n1: int, n2: int, n3: int) -> np.ndarray:
    g = g_vectors(recip, n1, n2, n3)
    return np.sqrt((g ** 2).sum(axis=-1))


# ----------------------------------------------------------------------------
# Cardinal B-spline ion-electron potential (CBSpline.f90, IonElectronSpline.f90)
# ----------------------------------------------------------------------------
def cardinal_bspline(order: int, x: float) -> np.ndarray:
    """M_n values on the integer offsets (GetCardinalBSpline, CBSpline.f90:42-98).

    Returns an array indexed 0..order; entry 0 stays zero."""
    s = np.zeros(order + 1)
    s[1] = x
    s[2] = 1.0 - x
    for n in range(3, order + 1):
        for k in range(0, n):
            s[n - k] = ((x + float(n - k - 1)) * s[n - k] + (float(k + 1) - x) * s[n - k - 1]) / float(n - 1)
    return s


def bspline_b(order: int, size: int, total: int) -> np.ndarray:
    """Euler exponential-spline factors b(m), m = 0..size-1 (FillB, CBSpline.f90:101-194)."""
    M = cardinal_bspline(order, 1.0)
    m = np.arange(size, dtype=float)
    k = np.arange(0, order - 1, dtype=float)
    denom = (M[1:order][None, :] * np.exp(2.0j * PI * m[:, None] * k[None, :] / float(total))).sum(axis=1)
    return np.exp(2.0j * PI * float(order - 1) * m / float(total)) / denom


def fill_q_ion_table(frac: np.ndarray, order: int, n1: int, n2: int, n3: int) -> np.ndarray:
    """Spread each ion on an order^3 B-spline stencil at -R (FillQIonTable, IonElectronSpline.f90:537-638)."""
    q = np.zeros((n1, n2, n3))
    for f in frac:
        gc = f * np.array([n1, n2, n3], dtype=float)
        fl = np.floor(gc)
        M1 = cardinal_bspline(order, gc[0] - fl[0])
        M2 = cardinal_bspline(order, gc[1] - fl[1])
        M3 = cardinal_bspline(order, gc[2] - fl[2])
        i = np.arange(order)
        l1 = np.mod(-int(fl[0]) + i, n1)
        l2 = np.mod(-int(fl[1]) + i, n2)
        l3 = np.mod(-int(fl[2]) + i, n3)
        w = M1[1:order + 1][:, None, None] * M2[1:order + 1][None, :, None] * M3[1:order + 1][None, None, :]
        np.add.at(q, (l1[:, None, None], l2[None, :, None], l3[None, None, :]), w)
    return q


def ion_potential_recip(cell: Cell, n1: int, n2: int, n3: int, order: int = SPLINE_ORDER) -> np.ndarray:
    """V_ion(G) on the half spectrum (IonElectronPotRecipSpline, IonElectronSpline.f90:83-216)."""
    k1 = n1 // 2 + 1
    qn = q_table(cell.recip, n1, n2, n3)
    acc = np.zeros((k1, n2, n3), dtype=complex)
    for s, sp in enumerate(cell.species):
        sel = cell.species_of_ion == s
        if not np.any(sel):
            continue
        qion = fill_q_ion_table(cell.frac[sel], order, n1, n2, n3)
        sf = fft_r2c(qion)
        acc += psp_lookup(sp, qn.ravel()).reshape(qn.shape) * sf
    b1 = bspline_b(order, k1, n1)
    b2 = bspline_b(order, n2, n2)
    b3 = bspline_b(order, n3, n3)
    tmp = acc * b1[:, None, None] * b2[None, :, None] * b3[None, None, :]
    return np.conj(tmp) / cell.vol * float(n1 * n2 * n3)


def ion_potential_real(cell: Cell, n1: int, n2: int, n3: int, order: int = SPLINE_ORDER) -> np.ndarray:
    """ionPotReal = backward FFT of V_ion(G) (RefreshIons.f90:215-221)."""
    return fft_c2r(ion_potential_recip(cell, n1, n2, n3, order), n1)


def uniform_density(cell: Cell, n1: int, n2: int, n3: int) -> np.ndarray:
    """rhoR = N_e / vol everywhere (System.f90:312-323)."""
    return np.full((n1, n2, n3), float(cell.num_electrons) / cell.vol)
