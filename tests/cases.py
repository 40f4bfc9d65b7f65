"""Test cases: the reference's golden cells (from tests/golden fixtures) and
small synthetic cells, set up through the oracle (which tests may import)."""
from __future__ import annotations

import json
import os

import numpy as np

from oracle import cellsetup as cs
from oracle import ewald as ew
from oracle import functional as fn
from oracle import kedf_kernels as kk
from oracle.consts import BOHR, HARTREE_TO_EV

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_ref_cases():
    with open(os.path.join(GOLDEN, "ref_cases.json")) as fh:
        return json.load(fh)


def al_species():
    z = np.load(os.path.join(GOLDEN, "al_hc_recpot.npz"))
    return cs.species_from_table(float(z["max_g"]), z["values"], "Al")


def cell_from_geometry(geom, species):
    lat = np.array(geom["lattice_angstrom_rows"], float).T / BOHR
    names = [s.name for s in species]
    frac = np.array([p[1:4] for p in geom["positions_frac"]], float)
    idx = np.array([names.index(p[0]) for p in geom["positions_frac"]], dtype=np.int64)
    return cs.Cell(lattice=lat, frac=frac, species_of_ion=idx, species=list(species))


def functional_for(cell, n, kinetic, alpha, beta, lam=1.0, mu=1.0, gamma=2.7, rho0=None, rho_s=None):
    n = tuple(int(x) for x in n)
    N = int(np.prod(n))
    dv = cell.vol / N
    qt = cs.q_table(cell.recip, *n)
    rho_avg = cell.num_electrons / cell.vol
    rho0 = rho_avg if rho0 is None else rho0
    rho_s = rho_avg if rho_s is None else rho_s
    if kinetic == fn.KEDF_WT:
        kern = kk.wt_kernel(qt, rho0, alpha, beta, lam, mu)[None]
    else:
        tabs = kk.wgc_radial_tables(alpha, beta, gamma)
        kern = kk.wgc_kernels(qt, rho_s, gamma, tabs)
    vion = cs.ion_potential_real(cell, *n)
    e_ii, _ = ew.ewald(cell.lattice, cell.frac, cell.charges())
    return fn.Functional(kinetic=kinetic, n=n, dv=dv, qtab=qt, kernel=kern, ion_pot=vion, ion_ion=e_ii,
                         lam=lam, mu=mu, alpha=alpha, beta=beta, rho_s=rho_s)


def golden_case(name):
    """(cell, functional, uniform density, case dict) for one reference run."""
    cases = load_ref_cases()
    c = cases[name]
    cell = cell_from_geometry(c["geometry"], [al_species()])
    n = cs.size_system(c["ecut_ev"] / HARTREE_TO_EV, cell.lattice)
    kin = fn.KEDF_WT if c["kinetic"] == "WT" else fn.KEDF_WGC
    f = functional_for(cell, n, kin, c["alpha"], c["beta"], c["lambda"], c["mu"], c.get("gamma", 2.7))
    return cell, f, cs.uniform_density(cell, *n), c


def random_density(n, ne, vol, seed=0, amp=0.3):
    """A smooth positive density with N_e electrons (for functional parity)."""
    rng = np.random.default_rng(seed)
    n1, n2, n3 = n
    x = np.arange(n1)[:, None, None] / n1
    y = np.arange(n2)[None, :, None] / n2
    z = np.arange(n3)[None, None, :] / n3
    f = np.ones(n)
    for _ in range(4):
        k = rng.integers(-2, 3, size=3)
        ph = rng.uniform(0, 2 * np.pi)
        f = f + amp * rng.uniform(0.2, 1.0) * np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + ph)
    f = np.abs(f) + 0.05
    f *= ne / (f.sum() * vol / f.size)
    return f


def engine_slot(eng, f, cell, precision=0):
    """Create a slot for oracle functional ``f`` and upload its tables."""
    s = eng.slot_create(f.n, cell.lattice, kinetic=f.kinetic, lam=f.lam, mu=f.mu, alpha=f.alpha, beta=f.beta,
                        rho0=0.0, rho_s=f.rho_s, ion_ion=f.ion_ion, precision=precision)
    eng.set_kernel(s, f.kernel)
    eng.set_ion_potential(s, f.ion_pot)
    return s


def oracle_cell(c):
    """Oracle cell of a synthetic workload cell (profess_b200.workloads.Cell):
    the same lattice, ions and Heine-Abarenkov tables."""
    from profess_b200 import workloads as wl
    sp = c.species[0]
    rc = 1.15 if sp.charge == 3 else 1.3
    mx, vals = wl.heine_abarenkov_table(float(sp.charge), rc, 0.1)
    return cs.Cell(lattice=c.lattice, frac=c.frac, species_of_ion=c.species_of_ion,
                   species=[cs.species_from_table(mx, vals, sp.name)])


def workload_functional(c):
    """(oracle cell, oracle functional) of a synthetic workload cell, with the
    product set-up's reference densities (rho0 = rho* = N_e / V)."""
    oc = oracle_cell(c)
    return oc, functional_for(oc, c.grid, c.kinetic, c.alpha, c.beta, gamma=c.gamma)
