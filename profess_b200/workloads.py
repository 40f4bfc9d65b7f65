"""Synthetic cells for the density-solve workloads (seeded).

All inputs are generated, none are read from a dataset:

* ``heine_abarenkov_species``: the bare Heine-Abarenkov model potential (V.
  Heine and I. Abarenkov, Phil. Mag. 9, 451 (1964)): a constant well of depth
  A inside the model radius r_c and the bare Coulomb tail -Z/r outside it.
  The benchmark configurations name a Goodwin-Heine-Abarenkov potential;
  these cells use the bare model potential that it is built on, without the
  Goodwin-Needs-Heine smoothing, with the configurations' Z, r_c and A.  Its
  transform is analytic, v(q) = -(4 pi / q^2) [Z cos(q r_c) + (A/q)(sin(q r_c)
  - q r_c cos(q r_c))], with the finite q -> 0 part 2 pi Z r_c^2 -
  4 pi A r_c^3 / 3 stored at q = 0.  It is tabulated as a recpot table (q
  spacing 0.002 bohr^-1 up to 30 bohr^-1, as in al_HC.lda.recpot), so the
  recpot reader's charge inference recovers Z from the -4 pi Z / q^2 tail.
  The shallow well keeps the valence density smooth at the cores, which the
  second-order WGC expansion needs.
* ``fcc_al``: FCC aluminium supercells of the 4-atom conventional cell.
* ``hcp_mg``: hexagonal magnesium supercells of the 2-atom primitive cell.
* ``Cell``: lattice (bohr, columns = lattice vectors), fractional positions,
  species table and the grid.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .recpot import BOHR, HARTREE_TO_EV, Species, species_from_table


@dataclasses.dataclass
class Cell:
    name: str
    lattice: np.ndarray        # (3, 3) bohr, column i = lattice vector i
    frac: np.ndarray           # (nion, 3)
    species_of_ion: np.ndarray  # (nion,)
    species: list
    grid: tuple
    kinetic: int = 4           # 4 WT, 5 WGC
    alpha: float = 5.0 / 6.0
    beta: float = 5.0 / 6.0
    gamma: float = 2.7

    @property
    def nion(self) -> int:
        return len(self.frac)

    @property
    def vol(self) -> float:
        return float(abs(np.linalg.det(self.lattice)))

    @property
    def num_electrons(self) -> int:
        return int(sum(self.species[s].charge for s in self.species_of_ion))

    def charges(self) -> np.ndarray:
        return np.array([self.species[s].charge for s in self.species_of_ion], dtype=float)


_HA_CACHE = {}


def heine_abarenkov_table(z: float, rc: float, a_well: float, dq: float = 0.002, npts: int = 15003):
    """(max_g in 1/A, values in eV*A^3) of the Heine-Abarenkov model potential."""
    key = (z, rc, a_well, dq, npts)
    if key in _HA_CACHE:
        return _HA_CACHE[key]
    q = np.arange(npts, dtype=float) * dq
    vals = np.empty(npts)
    vals[0] = 2.0 * math.pi * z * rc ** 2 - 4.0 * math.pi * a_well * rc ** 3 / 3.0
    qq = q[1:]
    x = qq * rc
    vals[1:] = -(4.0 * math.pi / qq ** 2) * (z * np.cos(x) + (a_well / qq) * (np.sin(x) - x * np.cos(x)))
    max_g_ang = (npts - 1) * dq / BOHR
    out = (max_g_ang, vals * BOHR ** 3 * HARTREE_TO_EV)
    _HA_CACHE[key] = out
    return out


def heine_abarenkov_species(name: str, z: int, rc: float, a_well: float = 0.1) -> Species:
    max_g, vals = heine_abarenkov_table(float(z), rc, a_well)
    return species_from_table(max_g, vals, name)


def al_species() -> Species:
    """Al: Z = 3, r_c = 1.15 bohr, A = 0.1 Ha."""
    return heine_abarenkov_species("Al", 3, 1.15, 0.1)


def mg_species() -> Species:
    """Mg: Z = 2, r_c = 1.3 bohr, A = 0.1 Ha."""
    return heine_abarenkov_species("Mg", 2, 1.3, 0.1)


def smooth_size(m: float) -> int:
    """Smallest 7-smooth integer >= m."""
    n = max(2, int(math.ceil(m - 1e-9)))
    while True:
        k = n
        for p in (2, 3, 5, 7):
            while k % p == 0:
                k //= p
        if k == 1:
            return n
        n += 1


def _displace(lat: np.ndarray, frac: np.ndarray, sigma_ang: float, rng) -> np.ndarray:
    d = rng.normal(0.0, sigma_ang / BOHR, size=frac.shape)        # cartesian, bohr
    return np.mod(frac + d @ np.linalg.inv(lat).T, 1.0)


def fcc_al(reps=(1, 1, 1), a_ang=4.05, sigma_ang=0.0, grid=None, seed=0, strain=0.0, pts_per_edge=24,
           kinetic=4) -> Cell:
    """FCC Al supercell of reps[0] x reps[1] x reps[2] conventional cells."""
    rng = np.random.default_rng(seed)
    a = a_ang * (1.0 + strain) / BOHR
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0, 0.5, 0.5], [0.5, 0, 0.5]], float)
    lat = np.diag([a * reps[0], a * reps[1], a * reps[2]])
    frac = np.concatenate([(basis + np.array([i, j, k], float)) / np.array(reps, float)
                           for i in range(reps[0]) for j in range(reps[1]) for k in range(reps[2])])
    if sigma_ang > 0:
        frac = _displace(lat, frac, sigma_ang, rng)
    if grid is None:
        grid = tuple(smooth_size(pts_per_edge * r) for r in reps)
    return Cell("fcc-Al-%dx%dx%d" % tuple(reps), lat, frac, np.zeros(len(frac), dtype=np.int64),
                [al_species()], tuple(grid), kinetic=kinetic)


def hcp_mg(reps=(8, 8, 9), a_ang=3.21, c_over_a=1.624, sigma_ang=0.0, grid=None, seed=0, kinetic=5,
           pts_per_ang=6.3) -> Cell:
    """hcp Mg supercell of the 2-atom hexagonal cell (a1 = a x, a2 = a(-1/2, sqrt3/2, 0), a3 = c z).
    The default 8 x 8 x 9 supercell has 1152 atoms."""
    rng = np.random.default_rng(seed)
    a = a_ang / BOHR
    c = a * c_over_a
    prim = np.array([[a, -0.5 * a, 0.0], [0.0, math.sqrt(3.0) / 2.0 * a, 0.0], [0.0, 0.0, c]])
    lat = prim * np.array(reps, float)[None, :]
    basis = np.array([[1.0 / 3.0, 2.0 / 3.0, 0.25], [2.0 / 3.0, 1.0 / 3.0, 0.75]])
    frac = np.concatenate([(basis + np.array([i, j, k], float)) / np.array(reps, float)
                           for i in range(reps[0]) for j in range(reps[1]) for k in range(reps[2])])
    if sigma_ang > 0:
        frac = _displace(lat, frac, sigma_ang, rng)
    if grid is None:
        lengths = np.sqrt((lat ** 2).sum(axis=0)) * BOHR
        grid = tuple(smooth_size(pts_per_ang * L) for L in lengths)
    alpha = (5.0 + math.sqrt(5.0)) / 6.0
    beta = (5.0 - math.sqrt(5.0)) / 6.0
    return Cell("hcp-Mg-%dx%dx%d" % tuple(reps), lat, frac, np.zeros(len(frac), dtype=np.int64),
                [mg_species()], tuple(grid), kinetic=kinetic, alpha=alpha if kinetic == 5 else 5.0 / 6.0,
                beta=beta if kinetic == 5 else 5.0 / 6.0)


def initial_density(cell: Cell, seed=0, noise=0.01) -> np.ndarray:
    """Uniform N_e/V times (1 + noise * U[0,1)), renormalised to N_e (Fortran order)."""
    rng = np.random.default_rng(seed + 7919)
    n = cell.grid
    rho = np.full(n, cell.num_electrons / cell.vol) * (1.0 + noise * rng.random(n))
    rho *= cell.num_electrons / (rho.sum() * cell.vol / rho.size)
    return np.asfortranarray(rho)


# ----------------------------------------------------------------- configs
def config_cell(cfg: int, seed: int = 0, index: int = 0) -> Cell:
    """The synthetic cell of one benchmark configuration.

    1: FCC Al 4 atoms, sigma 0.02 A, 32^3, WT.
    2: FCC Al 4x4x4 (256 atoms), sigma 0.05 A, 96^3, WT.
    3: FCC Al n x n x n, n ~ U{2..5}, a = 4.05 (1 +- 2%), 24 points per edge, WT.
    4: hcp Mg 8x8x9 (1152 atoms), sigma 0.05 A, 160x160x256, WGC."""
    if cfg == 1:
        return fcc_al((1, 1, 1), sigma_ang=0.02, grid=(32, 32, 32), seed=seed)
    if cfg == 2:
        return fcc_al((4, 4, 4), sigma_ang=0.05, grid=(96, 96, 96), seed=seed)
    if cfg == 3:
        rng = np.random.default_rng(seed * 1000 + index)
        n = int(rng.integers(2, 6))
        strain = float(rng.uniform(-0.02, 0.02))
        return fcc_al((n, n, n), sigma_ang=0.05, strain=strain, seed=seed * 1000 + index + 1)
    if cfg == 4:
        return hcp_mg((8, 8, 9), sigma_ang=0.05, grid=(160, 160, 256), seed=seed)
    raise ValueError("unknown config %r" % cfg)


def _near_cubic_reps(count: int, shape=(1.0, 1.0, 1.0)):
    """Integer supercell repeats with product close to count and lengths close to a cube."""
    best = None
    for a in range(1, 33):
        for b in range(1, 33):
            c = max(1, int(round(count / float(a * b))))
            if a * b * c == 0:
                continue
            lens = np.array([a * shape[0], b * shape[1], c * shape[2]])
            score = abs(a * b * c - count) / count + 0.3 * (lens.max() / lens.min() - 1.0)
            if best is None or score < best[0]:
                best = (score, (a, b, c))
    return best[1]


def serving_cell(rng) -> Cell:
    """One request of the serving mix: Al or Mg, atom count log-uniform in
    [32, 2048], KEDF 70% WT / 30% WGC, sigma ~ U[0.03, 0.1] A, grids 32-256
    points per axis (about 6 points per A, 7-smooth)."""
    species = "Al" if rng.random() < 0.5 else "Mg"
    natoms = float(np.exp(rng.uniform(np.log(32.0), np.log(2048.0))))
    kinetic = 4 if rng.random() < 0.7 else 5
    sigma = float(rng.uniform(0.03, 0.1))
    seed = int(rng.integers(1 << 30))
    if species == "Al":
        reps = _near_cubic_reps(max(1, int(round(natoms / 4.0))))
        cell = fcc_al(reps, sigma_ang=sigma, seed=seed, kinetic=kinetic)
    else:
        reps = _near_cubic_reps(max(1, int(round(natoms / 2.0))), shape=(1.0, 1.0, 1.624))
        cell = hcp_mg(reps, sigma_ang=sigma, seed=seed, kinetic=kinetic)
    lengths = np.sqrt((cell.lattice ** 2).sum(axis=0)) * BOHR
    cell.grid = tuple(min(256, max(32, smooth_size(5.9 * L))) for L in lengths)
    if kinetic == 5:
        cell.alpha = (5.0 + math.sqrt(5.0)) / 6.0
        cell.beta = (5.0 - math.sqrt(5.0)) / 6.0
    else:
        cell.alpha = cell.beta = 5.0 / 6.0
    return cell
