"""NVE, Nose-Hoover NVT and full-cell NPT molecular dynamics of many
independent cells (replicas) on one engine.

This is the reference's velocity-Verlet NVE driver, RunNVE
(Source/MolecularDynamicsNVE.f90:33-323), run for a batch of replicas in
lockstep.  Every step, for every replica: the centre-of-mass velocity is
removed and the centre of mass moved to the origin (MolecularDynamics.f90:
682-743, 1130-1191), a half kick, a drift, the ion terms are refreshed on the
device (B-spline ion potential, Ewald energy and forces), and
then the densities of all replicas are re-solved together by the engine's NTN
solver, warm-started from each replica's resident solution.  Forces follow
(ion-electron on the device, plus the Ewald forces) and a second half kick.

Units are atomic (bohr, Hartree, electron masses, a.u. of time).  The density
solves run in FP64 with the options given (the reference's density optimizer
settings); the positions, velocities and energies stay on the host.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import cell as pcell
from . import native
from .workloads import Cell

# Avogadro's number and the electron mass (g) as the reference stores them:
# single-precision literals held in double-precision parameters
# (Source/Constants.f90:60-61), hence the float32 rounding.
_MOL = float(np.float32(6.02214179e23))
_EMASS_G = float(np.float32(9.1093826e-28))
BOLTZMANN = 3.16682e-6              # Ha/K (Source/Constants.f90:65)
FUNDAMENTAL_TIME = 2.418884326505e-17  # s per a.u. of time (Source/Constants.f90:66)

# Standard atomic weights (g/mol) of AtomicMass (Source/Constants.f90:84+).
_ATOMIC_WEIGHT = {"H": 1.00794, "He": 4.002602, "Li": 6.9412, "Be": 9.012182, "B": 10.811, "C": 12.0107,
                  "N": 14.00674, "O": 15.9994, "F": 18.9984032, "Ne": 20.1797, "Na": 22.98976928,
                  "Mg": 24.3050, "Al": 26.981539, "Si": 28.0855, "P": 30.973762, "S": 32.066,
                  "Cl": 35.4527, "Ar": 39.948}


def atomic_mass(symbol: str) -> float:
    """Ion mass in electron masses, AtomicMass (Source/Constants.f90:84+)."""
    return _ATOMIC_WEIGHT[symbol.strip().capitalize()] / (_MOL * _EMASS_G)


def masses_of(cell: Cell) -> np.ndarray:
    return np.array([atomic_mass(cell.species[s].name) for s in cell.species_of_ion], dtype=float)


def initial_velocities(cell: Cell, temperature_k: float, seed: int = 0) -> np.ndarray:
    """Random velocities at a temperature, InitVelocity (MolecularDynamics.f90:575-679):
    Box-Muller normals divided by the mass, the centre-of-mass velocity removed,
    then scaled so that KE = 3/2 N k T.  The reference draws from the Fortran
    RANDOM_NUMBER generator; this one uses a seeded NumPy generator."""
    n = cell.nion
    m = masses_of(cell)
    rng = np.random.default_rng(seed)
    flat = np.zeros(3 * n)
    for i in range(1, 3 * n // 2 + 2):
        r1, r2 = rng.random(2)
        r1 = max(r1, np.finfo(float).tiny)
        a, b = np.sqrt(-2.0 * np.log(r1)) * np.cos(2 * np.pi * r2), np.sqrt(-2.0 * np.log(r1)) * np.sin(2 * np.pi * r2)
        if 2 * i - 2 < 3 * n:
            flat[2 * i - 2] = a
        if 2 * i - 1 < 3 * n:
            flat[2 * i - 1] = b
    v = flat.reshape(n, 3) / m[:, None]
    v -= (m[:, None] * v).sum(axis=0) / m.sum()
    ke = 0.5 * float((m[:, None] * v * v).sum())
    return v * np.sqrt(temperature_k * BOLTZMANN * 1.5 * n / ke)


@dataclasses.dataclass
class Replica:
    cell: Cell
    slot: int
    mass: np.ndarray
    vel: np.ndarray          # (nion, 3) bohr per a.u. of time
    cart: np.ndarray         # (nion, 3) unwrapped Cartesian positions (cartNoWrap)
    forces: np.ndarray = None
    f_ewald: np.ndarray = None   # Ewald forces of the current positions (host)
    energy: np.ndarray = None
    stats: dict = None
    history: list = dataclasses.field(default_factory=list)

    def kinetic_energy(self) -> float:
        return 0.5 * float((self.mass[:, None] * self.vel * self.vel).sum())

    def conserved(self) -> float:
        return self.kinetic_energy() + float(self.energy[0])

    def temperature(self) -> float:
        return 2.0 * self.kinetic_energy() / (3.0 * self.cell.nion) / BOLTZMANN


class NVE:
    """Lockstep NVE dynamics of ``cells`` (each gets one FP64 slot).

    ``dt`` in a.u. of time; ``velocities`` a list of (nion, 3) arrays (bohr per
    a.u. of time), or None for random ones at ``temperature_k``.
    ``opts``: NTN options of every density solve (native.ntn_options)."""

    def __init__(self, eng: native.Engine, cells, dt: float, velocities=None, temperature_k: float = 300.0,
                 seed: int = 0, opts=None, rho0=None):
        self.eng = eng
        self.dt = float(dt)
        self.opts = opts or native.ntn_options(conv_check=native.CONV_POT, pot_tol=1.0e-6)
        self.reps = []
        try:
            for k, c in enumerate(cells):
                c = dataclasses.replace(c, frac=np.array(c.frac, dtype=float))
                s = pcell.setup_slot(eng, c, native.FP64)
                v = (np.array(velocities[k], dtype=float) if velocities is not None
                     else initial_velocities(c, temperature_k, seed + k))
                self.reps.append(Replica(cell=c, slot=s, mass=masses_of(c), vel=v, cart=c.frac @ c.lattice.T))
            # the first solve starts from the given (or the uniform) density
            for k, r in enumerate(self.reps):
                self._refresh_ewald(r)
                rho = rho0[k] if rho0 is not None else np.full(r.cell.grid, r.cell.num_electrons / r.cell.vol)
                self.eng.start_solve(r.slot, np.asfortranarray(rho, dtype=float), self.opts)
            self._finish_solves()
        except Exception:
            self.close()
            raise

    def close(self):
        for r in self.reps:
            self.eng.slot_destroy(r.slot)
        self.reps = []

    # ------------------------------------------------------------------ steps
    def _refresh_ewald(self, r: Replica):
        """Ewald energy (into the slot's energy table) and forces of the positions
        of the slot's last ion-potential build, one device sum for both."""
        _, r.f_ewald = self.eng.ewald(r.slot, r.cell.nion)

    def _finish_solves(self):
        while self.eng.run(8):
            pass
        for r in self.reps:
            _, r.energy, r.stats = self.eng.result(r.slot, want_rho=False)
            if r.stats["outcome"] != 0:
                raise native.OfdftError(7, "density solve did not converge (replica slot %d)" % r.slot)
            r.forces = self.eng.forces(r.slot, r.cell.nion, include_ewald=False) + r.f_ewald

    def step(self):
        """One velocity-Verlet step of every replica (MolecularDynamicsNVE.f90:202-300)."""
        dt = self.dt
        for r in self.reps:
            c, m = r.cell, r.mass
            r.vel -= (m[:, None] * r.vel).sum(axis=0) / m.sum()          # RemoveMovementOfCenterOfMass
            linv = np.linalg.inv(c.lattice)
            r.cart -= (m[:, None] * r.cart).sum(axis=0) / m.sum()        # AdjustCenterOfMass
            c.frac = np.mod(r.cart @ linv.T, 1.0)
            r.vel += r.forces / m[:, None] * (0.5 * dt)
            r.cart += r.vel * dt
            c.frac = np.mod(c.frac + (r.vel * dt) @ linv.T, 1.0)
            # RefreshIonTerms: ion potential and Ewald sum on the device;
            # the density of the last solve is held on the device for the warm start
            self.eng.hold_density(r.slot)
            self.eng.build_ion_potential(r.slot, c.frac, c.species_of_ion, c.species)
            self._refresh_ewald(r)
            self.eng.start_solve(r.slot, None, self.opts)
        self._finish_solves()
        for r in self.reps:
            r.vel += r.forces / r.mass[:, None] * (0.5 * dt)
            r.history.append({"energy": float(r.energy[0]), "conserved": r.conserved(),
                              "temperature": r.temperature(), "num_evals": r.stats["num_evals"]})

    def run(self, nsteps: int):
        for _ in range(nsteps):
            self.step()


# ---------------------------------------------------------------------------- NVT
def yoshida_coefficients(n_yosh: int) -> np.ndarray:
    """Suzuki-Yoshida weights (MakeIntCoeff, MolecularDynamics.f90:506-540)."""
    if n_yosh == 1:
        return np.ones(1)
    if n_yosh == 3:
        w = np.full(3, 1.0 / (2.0 - 2.0 ** (1.0 / 3.0)))
        w[1] = 1.0 - 2.0 * w[1]
        return w
    if n_yosh == 5:
        w = np.full(5, 1.0 / (4.0 - 4.0 ** (1.0 / 3.0)))
        w[2] = 1.0 - 4.0 * w[2]
        return w
    raise ValueError("n_yosh must be 1, 3 or 5")


class NVT(NVE):
    """Lockstep Nose-Hoover NVT dynamics (RunNVT, Source/MolecularDynamicsNVT.f90:29-463):
    the NVE step with the thermostat integrated over a half step before the
    first kick and after the second (NHIntegrator: n_resn x n_yosh
    Suzuki-Yoshida substeps, thermostat mass ``q_mass``, target temperature
    ``temperature_k``).  The conserved quantity is KE + E + Q v_s^2 / 2 + g T x_s
    with g = 3 N degrees of freedom."""

    def __init__(self, eng, cells, dt: float, q_mass: float, temperature_k: float, velocities=None, seed: int = 0,
                 opts=None, rho0=None, n_resn: int = 3, n_yosh: int = 3):
        super().__init__(eng, cells, dt, velocities=velocities, temperature_k=temperature_k, seed=seed, opts=opts,
                         rho0=rho0)
        self.q_mass = float(q_mass)
        self.t_ha = float(temperature_k) * BOLTZMANN
        self.n_resn = int(n_resn)
        self.w = yoshida_coefficients(int(n_yosh))
        for r in self.reps:
            r.xlogs = 0.0
            r.vlogs = 0.0
            r.twice_ke = 2.0 * r.kinetic_energy()

    def _thermostat(self, r):
        """NHIntegrator (MolecularDynamicsNVT.f90:322-399)."""
        g = 3.0 * r.cell.nion
        scaling = 1.0
        glogs = (r.twice_ke - g * self.t_ha) / self.q_mass
        for _ in range(self.n_resn):
            for w in self.w:
                wdt2 = w * self.dt / (2.0 * self.n_resn)
                wdt4 = w * self.dt / (4.0 * self.n_resn)
                r.vlogs += glogs * wdt4
                scaling *= np.exp(-wdt2 * r.vlogs)
                glogs = (scaling * scaling * r.twice_ke - g * self.t_ha) / self.q_mass
                r.xlogs += r.vlogs * wdt2
                r.vlogs += glogs * wdt4
        r.vel *= scaling
        r.twice_ke *= scaling * scaling

    def conserved_nh(self, r) -> float:
        g = 3.0 * r.cell.nion
        return 0.5 * r.twice_ke + float(r.energy[0]) + 0.5 * r.vlogs ** 2 * self.q_mass + g * self.t_ha * r.xlogs

    def step(self):
        """One NVT step of every replica (MolecularDynamicsNVT.f90:201-300)."""
        dt = self.dt
        for r in self.reps:
            c, m = r.cell, r.mass
            r.vel -= (m[:, None] * r.vel).sum(axis=0) / m.sum()
            linv = np.linalg.inv(c.lattice)
            r.cart -= (m[:, None] * r.cart).sum(axis=0) / m.sum()
            c.frac = np.mod(r.cart @ linv.T, 1.0)
            self._thermostat(r)   # with the kinetic energy of the end of the last step, as the reference
            r.vel += r.forces / m[:, None] * (0.5 * dt)
            r.cart += r.vel * dt
            c.frac = np.mod(c.frac + (r.vel * dt) @ linv.T, 1.0)
            self.eng.hold_density(r.slot)
            self.eng.build_ion_potential(r.slot, c.frac, c.species_of_ion, c.species)
            self._refresh_ewald(r)
            self.eng.start_solve(r.slot, None, self.opts)
        self._finish_solves()
        for r in self.reps:
            r.vel += r.forces / r.mass[:, None] * (0.5 * dt)
            r.twice_ke = 2.0 * r.kinetic_energy()
            self._thermostat(r)
            r.history.append({"energy": float(r.energy[0]), "conserved": self.conserved_nh(r),
                              "temperature": r.temperature(), "num_evals": r.stats["num_evals"]})


# ---------------------------------------------------------------------------- NPT
def box_constraint(m: np.ndarray, constr_type: int) -> np.ndarray:
    """BoxConstraint (Source/MolecularDynamicsNPT.f90:878-935) on a 3x3 box
    force or velocity: -1 none, 1 orthogonal box, 3/4/5 x/y/z fixed and
    orthogonal."""
    m = np.array(m, dtype=float)
    if constr_type < 0:
        return m
    if constr_type == 1:
        return np.diag(np.diag(m))
    if constr_type in (3, 4, 5):
        m = np.diag(np.diag(m))
        m[constr_type - 3, constr_type - 3] = 0.0
        return m
    raise ValueError("box constraint type %d is not implemented" % constr_type)


def _sym_exp(m: np.ndarray, scale: float) -> np.ndarray:
    """V diag(exp(scale * eig)) V^T of a symmetric 3x3 matrix (Diag, DSPEV on
    the upper triangle, Source/MathFunctions.f90:762-811)."""
    eig, v = np.linalg.eigh(m, UPLO="U")
    return v @ np.diag(np.exp(scale * eig)) @ v.T


class NPT(NVE):
    """Lockstep full-cell NPT dynamics (NPTFullCell, Source/MolecularDynamicsNPT.f90:76-274):
    the Martyna-Tobias-Klein integrator with a Nose-Hoover thermostat
    (``q_mass``) and a barostat (``b_mass``) at external pressure ``ext_pres``
    (Ha/bohr^3).  Each step: NPTFullCell_Integrator over a half step, MVV
    (a half kick, the positions and the lattice propagated by the barostat
    velocity, RefreshCellSetup on the device: new lattice, kinetic kernel, ion
    potential and Ewald sum; RescaleDensity of the held density; the density
    solves of all replicas together; forces, stress and a half kick), and the
    integrator again.  The stress is the device stress of each new density.
    WT or second-order WGC cells."""

    def __init__(self, eng, cells, dt: float, q_mass: float, b_mass: float, temperature_k: float,
                 ext_pres: float, velocities=None, seed: int = 0, opts=None, rho0=None, n_resn: int = 3,
                 n_yosh: int = 3, constr_type: int = -1):
        self.q_mass, self.b_mass = float(q_mass), float(b_mass)
        self.t_ha = float(temperature_k) * BOLTZMANN
        self.ext_pres = float(ext_pres)
        self.n_resn = int(n_resn)
        self.w = yoshida_coefficients(int(n_yosh))
        self.constr = int(constr_type)
        shifted, carts = [], []
        for c in cells:  # AdjustCenterOfMass(.TRUE.) before the set-up
            c = dataclasses.replace(c, frac=np.array(c.frac, dtype=float), lattice=np.array(c.lattice, float))
            m = masses_of(c)
            cart = c.frac @ c.lattice.T
            cart -= (m[:, None] * cart).sum(axis=0) / m.sum()
            c.frac = np.mod(cart @ np.linalg.inv(c.lattice).T, 1.0)
            shifted.append(c)
            carts.append(cart)
        super().__init__(eng, shifted, dt, velocities=velocities, temperature_k=temperature_k, seed=seed,
                         opts=opts, rho0=rho0)
        for r, cart in zip(self.reps, carts):
            r.cart = cart  # unwrapped (cartNoWrap)
            r.xlogs, r.vlogs = 0.0, 0.0
            r.vboxg = box_constraint(np.zeros((3, 3)), self.constr)
            r.stress = self.eng.stress(r.slot)
            r.freedom = 3.0 * r.cell.nion

    # ------------------------------------------------------------ pieces
    def _ke(self, r):
        return 0.5 * float((r.mass[:, None] * r.vel * r.vel).sum())

    def _ke_tensor(self, r):
        return 0.5 * (r.mass[:, None] * r.vel).T @ r.vel

    def _box_ke(self, r):
        return 0.5 * self.b_mass * float((r.vboxg ** 2).sum())

    def _g_box(self, r, ke, ket, pint):
        g = (2.0 * ket + r.cell.vol * pint) / self.b_mass
        g += np.eye(3) * (2.0 * ke / r.freedom - r.cell.vol * self.ext_pres) / self.b_mass
        return box_constraint(g, self.constr)

    def _integrator(self, r):
        """NPTFullCell_Integrator (MolecularDynamicsNPT.f90:413-640)."""
        T, Q, f = self.t_ha, self.q_mass, r.freedom
        ke, ket, boxke = self._ke(r), self._ke_tensor(r), self._box_ke(r)
        glogs = (2.0 * ke + 2.0 * boxke - (f + 9.0) * T) / Q
        pint = -r.stress
        gbox = self._g_box(r, ke, ket, pint)
        for _ in range(self.n_resn):
            for w in self.w:
                wdt2 = w * self.dt / (2.0 * self.n_resn)
                wdt4 = w * self.dt / (4.0 * self.n_resn)
                wdt8 = w * self.dt / (8.0 * self.n_resn)
                r.vlogs += glogs * wdt4
                aa = np.exp(-wdt8 * r.vlogs)
                r.vboxg = r.vboxg * aa * aa + wdt4 * gbox * aa
                vt = r.vboxg + np.eye(3) * (np.trace(r.vboxg) / f + r.vlogs)
                r.vel = r.vel @ _sym_exp(vt, -wdt2).T
                r.xlogs += r.vlogs * wdt2
                ke, ket = self._ke(r), self._ke_tensor(r)
                gbox = self._g_box(r, ke, ket, pint)
                aa = np.exp(-wdt8 * r.vlogs)
                r.vboxg = r.vboxg * aa * aa + wdt4 * gbox * aa
                boxke = self._box_ke(r)
                glogs = (2.0 * ke + 2.0 * boxke - (f + 9.0) * T) / Q
                r.vlogs += glogs * wdt4

    def conserved_npt(self, r) -> float:
        """NPTFullCell_Conserved (MolecularDynamicsNPT.f90:691-790)."""
        return (self._ke(r) + float(r.energy[0]) + self.ext_pres * r.cell.vol + self._box_ke(r) +
                0.5 * r.vlogs ** 2 * self.q_mass + (r.freedom + 9.0) * self.t_ha * r.xlogs)

    def step(self):
        """One NPT step of every replica (MolecularDynamicsNPT.f90:226-265)."""
        dt, dt2 = self.dt, 0.5 * self.dt
        for r in self.reps:
            self._integrator(r)
            # MVV (MolecularDynamicsNPT.f90:275-411)
            r.vel += dt2 * r.forces / r.mass[:, None]
            eig, v = np.linalg.eigh(r.vboxg, UPLO="U")
            arg2 = (eig * dt2) ** 2
            poly = 1.0 + arg2 / 6.0 + arg2 ** 2 / 120.0 + arg2 ** 3 / 5040.0 + arg2 ** 4 / 362880.0
            vt1 = v @ np.diag(np.exp(dt * eig)) @ v.T
            vt2 = v @ np.diag(np.exp(dt2 * eig) * poly) @ v.T
            r.cart = r.cart @ vt1.T + dt * r.vel @ vt2.T
            lat = vt1 @ r.cell.lattice
            lat = _symmetrize(lat)
            c = r.cell
            c.lattice = lat
            c.frac = np.mod(r.cart @ np.linalg.inv(lat).T, 1.0)
            # RefreshCellSetup and RescaleDensity on the device, then the solve
            self.eng.hold_density(r.slot)
            rho_avg = c.num_electrons / c.vol
            self.eng.set_lattice(r.slot, lat, rho_avg, rho_avg)
            self.eng.rescale_input(r.slot, c.num_electrons)
            pcell.build_kernel(self.eng, r.slot, c)
            self.eng.build_ion_potential(r.slot, c.frac, c.species_of_ion, c.species)
            self._refresh_ewald(r)
            self.eng.start_solve(r.slot, None, self.opts)
        self._finish_solves()
        for r in self.reps:
            r.stress = self.eng.stress(r.slot)
            r.vel += dt2 * r.forces / r.mass[:, None]
            self._integrator(r)
            r.history.append({"energy": float(r.energy[0]), "conserved": self.conserved_npt(r),
                              "volume": r.cell.vol, "temperature": r.temperature(),
                              "num_evals": r.stats["num_evals"]})


def _symmetrize(a: np.ndarray) -> np.ndarray:
    """Symmetrize (Source/MathFunctions.f90:813-850): off-diagonal pairs averaged."""
    return 0.5 * (a + a.T)
