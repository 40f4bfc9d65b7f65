"""Test infrastructure (the oracle): a CPU restatement of the reference's NVE
molecular dynamics, RunNVE (Source/MolecularDynamicsNVE.f90:33-323), and of
its Nose-Hoover NVT variant, RunNVT (Source/MolecularDynamicsNVT.f90:29-463),
on the oracle's functional, NTN solver and forces.  Only tests import it.

Per step: RemoveMovementOfCenterOfMass (MolecularDynamics.f90:682-743),
AdjustCenterOfMass with the shift (MolecularDynamics.f90:1130-1191), half
kick, drift of the unwrapped Cartesian and the wrapped fractional positions
(MolecularDynamicsNVE.f90:208-229), RefreshIonTerms (ion potential and Ewald
energy for the new positions), the density solve warm-started from the last
density, CalculateForces, half kick, and the conserved energy KE + E_total
(Conserved, MolecularDynamicsNVE.f90:378-425).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import cellsetup as cs
from . import ewald as ew
from . import forces as ofo
from . import functional as fn
from . import kedf_kernels as kk
from . import ntn

# AtomicMass (Source/Constants.f90:84+): g/mol over Avogadro's number times the
# electron mass, both single-precision literals in the reference
# (Source/Constants.f90:60-61).
_MOL = float(np.float32(6.02214179e23))
_EMASS = float(np.float32(9.1093826e-28))
_WEIGHT = {"Al": 26.981539, "Mg": 24.3050}


def atomic_mass(symbol: str) -> float:
    return _WEIGHT[symbol] / (_MOL * _EMASS)


_WGC_TABS = {}


def functional_for(cell: cs.Cell, n, alpha: float, beta: float, kinetic: int = fn.KEDF_WT,
                   gamma: float = 2.7) -> fn.Functional:
    """The WT (or second-order WGC) functional of ``cell`` on grid n, its
    kernel built at rho0 = rho* = N/V, with the B-spline ion potential and the
    Ewald energy of its current positions (RefreshIonTerms,
    Source/RefreshIons.f90:125-238).  The WGC radial tables depend only on
    (alpha, beta, gamma) and are integrated once."""
    n = tuple(int(x) for x in n)
    qt = cs.q_table(cell.recip, *n)
    rho_avg = cell.num_electrons / cell.vol
    if kinetic == fn.KEDF_WT:
        kern = kk.wt_kernel(qt, rho_avg, alpha, beta, 1.0, 1.0)[None]
    else:
        key = (float(alpha), float(beta), float(gamma))
        if key not in _WGC_TABS:
            _WGC_TABS[key] = kk.wgc_radial_tables(alpha, beta, gamma)
        kern = kk.wgc_kernels(qt, rho_avg, gamma, _WGC_TABS[key])
    vion = cs.ion_potential_real(cell, *n)
    e_ii, _ = ew.ewald(cell.lattice, cell.frac, cell.charges())
    return fn.Functional(kinetic=kinetic, n=n, dv=cell.vol / float(np.prod(n)), qtab=qt, kernel=kern,
                         ion_pot=vion, ion_ion=e_ii, lam=1.0, mu=1.0, alpha=alpha, beta=beta, rho_s=rho_avg)


@dataclasses.dataclass
class NveState:
    frac: np.ndarray
    cart: np.ndarray
    vel: np.ndarray
    rho: np.ndarray
    forces: np.ndarray
    energy: float
    conserved: float


def run_nve(cell: cs.Cell, n, vel0: np.ndarray, dt: float, nsteps: int, opts: ntn.NtnOptions,
            alpha: float = 5.0 / 6.0, beta: float = 5.0 / 6.0, rho0=None):
    """Returns the list of states after the initial solve and after each step."""
    cell = dataclasses.replace(cell, frac=np.array(cell.frac, dtype=float))
    m = np.array([atomic_mass(cell.species[s].name) for s in cell.species_of_ion])
    linv = np.linalg.inv(cell.lattice)
    rho = cs.uniform_density(cell, *n) if rho0 is None else rho0
    f = functional_for(cell, n, alpha, beta)
    r = ntn.NtnSolver(f, opts).solve(rho)
    rho = r.rho
    forces, _, _ = ofo.total_forces(cell, rho)
    vel = np.array(vel0, dtype=float)
    cart = cell.frac @ cell.lattice.T
    ke = lambda v: 0.5 * float((m[:, None] * v * v).sum())
    out = [NveState(cell.frac.copy(), cart.copy(), vel.copy(), rho, forces, float(r.energy[0]),
                    ke(vel) + float(r.energy[0]))]
    for _ in range(nsteps):
        vel = vel - (m[:, None] * vel).sum(axis=0) / m.sum()
        cart = cart - (m[:, None] * cart).sum(axis=0) / m.sum()
        cell.frac = np.mod(cart @ linv.T, 1.0)
        vel = vel + forces / m[:, None] * (0.5 * dt)
        cart = cart + vel * dt
        cell.frac = np.mod(cell.frac + (vel * dt) @ linv.T, 1.0)
        f = functional_for(cell, n, alpha, beta)
        r = ntn.NtnSolver(f, opts).solve(rho)
        rho = r.rho
        forces, _, _ = ofo.total_forces(cell, rho)
        vel = vel + forces / m[:, None] * (0.5 * dt)
        out.append(NveState(cell.frac.copy(), cart.copy(), vel.copy(), rho, forces, float(r.energy[0]),
                            ke(vel) + float(r.energy[0])))
    return out


def _yoshida(n):
    if n == 1:
        return np.ones(1)
    if n == 3:
        w = np.full(3, 1.0 / (2.0 - 2.0 ** (1.0 / 3.0)))
        w[1] = 1.0 - 2.0 * w[1]
        return w
    w = np.full(5, 1.0 / (4.0 - 4.0 ** (1.0 / 3.0)))
    w[2] = 1.0 - 4.0 * w[2]
    return w


def run_nvt(cell: cs.Cell, n, vel0: np.ndarray, dt: float, nsteps: int, opts: ntn.NtnOptions, q_mass: float,
            temperature_ha: float, n_resn: int = 3, n_yosh: int = 3, alpha: float = 5.0 / 6.0,
            beta: float = 5.0 / 6.0):
    """Nose-Hoover NVT, RunNVT and NHIntegrator (Source/MolecularDynamicsNVT.f90:29-463, 322-399).
    Returns the list of (frac, vel, energy, conserved) after each step."""
    cell = dataclasses.replace(cell, frac=np.array(cell.frac, dtype=float))
    m = np.array([atomic_mass(cell.species[s].name) for s in cell.species_of_ion])
    linv = np.linalg.inv(cell.lattice)
    g = 3.0 * len(m)
    w = _yoshida(n_yosh)
    rho = cs.uniform_density(cell, *n)
    r = ntn.NtnSolver(functional_for(cell, n, alpha, beta), opts).solve(rho)
    rho = r.rho
    energy = float(r.energy[0])
    forces, _, _ = ofo.total_forces(cell, rho)
    vel = np.array(vel0, dtype=float)
    cart = cell.frac @ cell.lattice.T
    st = {"x": 0.0, "v": 0.0, "k2": float((m[:, None] * vel * vel).sum())}

    def thermostat(vel):
        scaling = 1.0
        gl = (st["k2"] - g * temperature_ha) / q_mass
        for _ in range(n_resn):
            for wi in w:
                wdt2 = wi * dt / (2.0 * n_resn)
                wdt4 = wi * dt / (4.0 * n_resn)
                st["v"] += gl * wdt4
                scaling *= np.exp(-wdt2 * st["v"])
                gl = (scaling ** 2 * st["k2"] - g * temperature_ha) / q_mass
                st["x"] += st["v"] * wdt2
                st["v"] += gl * wdt4
        st["k2"] *= scaling ** 2
        return vel * scaling

    out = []
    for _ in range(nsteps):
        vel = vel - (m[:, None] * vel).sum(axis=0) / m.sum()
        cart = cart - (m[:, None] * cart).sum(axis=0) / m.sum()
        cell.frac = np.mod(cart @ linv.T, 1.0)
        vel = thermostat(vel)
        vel = vel + forces / m[:, None] * (0.5 * dt)
        cart = cart + vel * dt
        cell.frac = np.mod(cell.frac + (vel * dt) @ linv.T, 1.0)
        r = ntn.NtnSolver(functional_for(cell, n, alpha, beta), opts).solve(rho)
        rho = r.rho
        energy = float(r.energy[0])
        forces, _, _ = ofo.total_forces(cell, rho)
        vel = vel + forces / m[:, None] * (0.5 * dt)
        st["k2"] = float((m[:, None] * vel * vel).sum())
        vel = thermostat(vel)
        h = 0.5 * st["k2"] + energy + 0.5 * st["v"] ** 2 * q_mass + g * temperature_ha * st["x"]
        out.append((cell.frac.copy(), vel.copy(), energy, h))
    return out


def run_npt(cell: cs.Cell, n, vel0: np.ndarray, dt: float, nsteps: int, opts: ntn.NtnOptions, q_mass: float,
            b_mass: float, temperature_ha: float, ext_pres: float, n_resn: int = 3, n_yosh: int = 3,
            alpha: float = 5.0 / 6.0, beta: float = 5.0 / 6.0, kinetic: int = fn.KEDF_WT, gamma: float = 2.7):
    """Full-cell NPT, NPTFullCell / MVV / NPTFullCell_Integrator / NPTFullCell_Conserved
    (Source/MolecularDynamicsNPT.f90:76-274, 275-411, 413-640, 691-790), no box
    constraint and no frozen ions.  Velocities are held (3, numIon) as in the
    reference.  kinetic = KEDF_WGC runs the second-order WGC functional.
    Returns the list of (lattice, frac, energy, conserved, volume) after the
    first solve and after each step."""
    from . import stress as ost
    cell = dataclasses.replace(cell, frac=np.array(cell.frac, dtype=float), lattice=np.array(cell.lattice, float))
    mass = np.array([atomic_mass(cell.species[s].name) for s in cell.species_of_ion])
    nion = len(mass)
    freedom = 3.0 * nion
    d = 3.0
    w = _yoshida(n_yosh)
    vel = np.array(vel0, dtype=float).T.copy()            # (3, numIon)
    cart = np.array([cell.lattice @ cell.frac[i] for i in range(nion)]).T   # cartNoWrap (3, numIon)
    com = (cart * mass[None, :]).sum(axis=1) / mass.sum()  # AdjustCenterOfMass(.TRUE.)
    cart = cart - com[:, None]
    inv = np.linalg.inv(cell.lattice)
    cell.frac = np.array([np.mod(inv @ cart[:, i], 1.0) for i in range(nion)])
    xlogs = vlogs = 0.0
    vbox = np.zeros((3, 3))

    def refresh_and_solve(rho):
        f = functional_for(cell, n, alpha, beta, kinetic, gamma)
        r = ntn.NtnSolver(f, opts).solve(rho)
        forces, _, _ = ofo.total_forces(cell, r.rho)
        return r.rho, float(r.energy[0]), forces, ost.stress(cell, f, r.rho, gamma=gamma)

    rho, energy, forces, stress = refresh_and_solve(cs.uniform_density(cell, *n))

    def atom_ke():
        return sum(0.5 * mass[i] * float(vel[:, i] @ vel[:, i]) for i in range(nion))

    def atom_ke_tensor():
        t = np.zeros((3, 3))
        for a in range(3):
            for b in range(3):
                t[a, b] = sum(0.5 * mass[i] * vel[a, i] * vel[b, i] for i in range(nion))
        return t

    def box_ke():
        return 0.5 * b_mass * float((vbox ** 2).sum())

    def diag_exp(m, scale):
        eig, v = np.linalg.eigh(m, UPLO="U")
        return v @ np.diag(np.exp(scale * eig)) @ v.T

    def integrator():
        nonlocal vlogs, xlogs, vbox, vel
        ke, ket = atom_ke(), atom_ke_tensor()
        glogs = (2.0 * ke + 2.0 * box_ke() - (freedom + 3.0 ** 2) * temperature_ha) / q_mass
        pint = -stress
        gbox = (2.0 * ket + cell.vol * pint) / b_mass
        gbox = gbox + np.eye(3) * (2.0 * ke / freedom - cell.vol * ext_pres) / b_mass
        for _ in range(n_resn):
            for wi in w:
                wdt2 = wi * dt / (2.0 * n_resn)
                wdt4 = wi * dt / (4.0 * n_resn)
                wdt8 = wi * dt / (8.0 * n_resn)
                vlogs = vlogs + glogs * wdt4
                aa = np.exp(-wdt8 * vlogs)
                vbox = vbox * aa * aa + wdt4 * gbox * aa
                trvg = (vbox[0, 0] + vbox[1, 1] + vbox[2, 2]) / freedom
                vt = vbox.copy()
                for k in range(3):
                    vt[k, k] += trvg + vlogs
                vt = diag_exp(vt, -wdt2)
                for i in range(nion):
                    vel[:, i] = vt @ vel[:, i]
                xlogs = xlogs + vlogs * wdt2
                ke, ket = atom_ke(), atom_ke_tensor()
                gbox = (2.0 * ket + cell.vol * pint) / b_mass
                gbox = gbox + np.eye(3) * (2.0 * ke / freedom - cell.vol * ext_pres) / b_mass
                aa = np.exp(-wdt8 * vlogs)
                vbox = vbox * aa * aa + wdt4 * gbox * aa
                glogs = (2.0 * ke + 2.0 * box_ke() - (freedom + 3.0 ** 2) * temperature_ha) / q_mass
                vlogs = vlogs + glogs * wdt4

    def conserved():
        return (atom_ke() + energy + ext_pres * cell.vol + box_ke() + 0.5 * vlogs ** 2 * q_mass +
                (freedom + d ** 2) * temperature_ha * xlogs)

    out = [(cell.lattice.copy(), cell.frac.copy(), energy, conserved(), cell.vol)]
    for _ in range(nsteps):
        integrator()
        dt2 = dt / 2.0
        for i in range(nion):
            vel[:, i] = vel[:, i] + dt2 * forces[i, :] / mass[i]
        eig, v = np.linalg.eigh(vbox, UPLO="U")
        ie = np.diag(np.exp(dt * eig))
        arg2 = (eig * dt2) ** 2
        poly = 1.0 + arg2 / 6.0 + arg2 ** 2 / 120.0 + arg2 ** 3 / 5040.0 + arg2 ** 4 / 362880.0
        is_ = np.diag(np.exp(dt2 * eig) * poly)
        vt1 = v @ (ie @ v.T)
        vt2 = v @ (is_ @ v.T)
        for i in range(nion):
            cart[:, i] = vt1 @ cart[:, i] + dt * (vt2 @ vel[:, i])
        lat = vt1 @ cell.lattice
        sym = lat.copy()
        for a in range(3):
            for b in range(3):
                if a != b:
                    sym[a, b] = (lat[a, b] + lat[b, a]) / 2.0
        cell.lattice = sym
        inv = np.linalg.inv(cell.lattice)
        cell.frac = np.array([np.mod(inv @ cart[:, i], 1.0) for i in range(nion)])
        rho = rho * (cell.num_electrons / (rho.sum() * cell.vol / rho.size))   # RescaleDensity
        rho, energy, forces, stress = refresh_and_solve(rho)
        for i in range(nion):
            vel[:, i] = vel[:, i] + dt2 * forces[i, :] / mass[i]
        integrator()
        out.append((cell.lattice.copy(), cell.frac.copy(), energy, conserved(), cell.vol))
    return out
