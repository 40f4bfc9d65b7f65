"""Put a cell on an engine slot with every table built by the library.

This is the set-up the reference does before its first density solve
(Source/Initializer.f90; KEDFRefresh, Source/SetupKEDF.f90:629-683;
RefreshIonTerms, Source/RefreshIons.f90:125-238): the kinetic kernel is
filled on the device (WT from LindG, WGC from the kernel ODE's radial tables),
the ion-electron potential is built on the device by the B-spline method and
the Ewald energy is summed on the host.
"""
from __future__ import annotations

from . import native
from .workloads import Cell


def ion_ion_energy(lib, cell: Cell) -> float:
    e, _ = native.ewald(lib, cell.lattice, cell.frac, cell.charges())
    return e


_WGC_TABLES = {}


def wgc_tables(lib, alpha: float, beta: float, gamma: float):
    """Radial WGC kernel tables, integrated once per (alpha, beta, gamma) and kept."""
    key = (float(alpha), float(beta), float(gamma))
    if key not in _WGC_TABLES:
        _WGC_TABLES[key] = native.wgc_radial_tables(lib, *key)
    return _WGC_TABLES[key]


def build_kernel(eng: native.Engine, slot: int, cell: Cell) -> None:
    """Build the slot's kinetic kernel on the device at its current rho0 and
    rho* (WT: the LindG kernel; second-order WGC: the kernel planes from the
    radial tables of (alpha, beta, gamma)), as RefreshCellSetup does after a
    lattice change."""
    if cell.kinetic == native.KEDF_WT:
        eng.build_wt_kernel(slot)
    else:
        eng.build_wgc_kernel(slot, wgc_tables(eng.lib, cell.alpha, cell.beta, cell.gamma))


def _create(eng: native.Engine, cell: Cell, precision, ion_ion) -> int:
    rho_avg = cell.num_electrons / cell.vol
    return eng.slot_create(cell.grid, cell.lattice, kinetic=cell.kinetic, alpha=cell.alpha, beta=cell.beta,
                           gamma=cell.gamma, rho0=rho_avg, rho_s=rho_avg, ion_ion=ion_ion, precision=precision)


def slot_like(eng: native.Engine, cell: Cell, src: int, precision=native.FP32) -> int:
    """A slot for ``cell`` whose kernel planes, ion potential and ion-ion
    energy are converted on the device from slot ``src`` (already set up for
    the same cell): the second precision of a mixed-precision request."""
    s = _create(eng, cell, precision, 0.0)
    try:
        eng.copy_tables(s, src)
    except Exception:
        eng.slot_destroy(s)
        raise
    return s


def setup_slot(eng: native.Engine, cell: Cell, precision=native.FP64, ion_ion=None) -> int:
    """Create a slot for ``cell`` and build its kernel and ion potential on the
    device; the Ewald energy is summed on the device unless ``ion_ion`` gives it."""
    s = _create(eng, cell, precision, 0.0 if ion_ion is None else ion_ion)
    try:
        build_kernel(eng, s, cell)
        eng.build_ion_potential(s, cell.frac, cell.species_of_ion, cell.species)
        if ion_ion is None:
            eng.ewald(s, cell.nion, want_forces=False)
    except Exception:
        eng.slot_destroy(s)
        raise
    return s
