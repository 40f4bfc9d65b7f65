"""The benchmark cells at full size through the product set-up path, against
the FP64 oracle (GPU).

Every cell is built the way ``bench.py`` and the serving layer build it
(``profess_b200.cell.setup_slot``: the kinetic kernel filled on the device,
the B-spline ion-electron potential spread and transformed on the device, the
Ewald energy summed on the device), and the oracle builds the same cell from
the same tables on the host.  At a fixed non-uniform density one evaluation
is compared term by term with the oracle's ``CalculatePotentialPlus``
(Source/CalPotential.f90:610-644 energy table), together with the potential
and the ion forces (Source/CalForce.f90:36-73).

Bounds (Hartree atomic units):
* FP64 slots: every energy term within 1e-8 Ha/atom, potential RMS within
  1e-7, forces within 1e-7 Ha/bohr, the ion potential within 1e-9 Ha.
* FP32 slots: every energy term within 1e-5 eV/atom, the potential RMS
  within 1e-5 Ha (the potential is the small sum of large cancelling terms,
  so its FP32 error is stated absolutely; measured 1.3e-6 to 2.1e-6).
* cfg2 FP64 NTN solve to potNorm < 1e-6: the energy terms within 1e-8
  Ha/atom of the oracle's solve and the forces on the two converged
  densities within 1e-7 Ha/bohr.
"""
import numpy as np
import pytest

import cases
from oracle import forces as ofo
from oracle import functional as fn
from oracle import ntn
from oracle.consts import HARTREE_TO_EV
from profess_b200 import cell as pcell
from profess_b200 import native, workloads as wl

pytestmark = pytest.mark.gpu

# name -> the workload cell: cfg2 (256-atom Al, 96^3), the smallest and the
# largest cfg3 grids of the bench's first batch (32 atoms at 48^3, 500 atoms
# at 120^3) and cfg4 (1152-atom hcp Mg, 160x160x256, WGC)
CELLS = {
    "cfg2": lambda: wl.config_cell(2, seed=0),
    "cfg3_48": lambda: wl.config_cell(3, seed=1, index=13),
    "cfg3_120": lambda: wl.config_cell(3, seed=1, index=1),
    "cfg4": lambda: wl.config_cell(4, seed=0),
}

_ORACLE = {}


def oracle_case(name):
    """(workload cell, oracle cell, oracle functional, density, oracle potential,
    oracle energies, oracle forces), computed once per cell."""
    if name not in _ORACLE:
        c = CELLS[name]()
        oc, f = cases.workload_functional(c)
        rho = cases.random_density(c.grid, oc.num_electrons, oc.vol, seed=11, amp=0.1)
        pot, et = fn.calculate_potential_plus(f, rho)
        F, _, _ = ofo.total_forces(oc, rho)
        _ORACLE[name] = (c, oc, f, rho, pot, et, F)
    return _ORACLE[name]


def _report(name, prec, nat, et_g, et_o, pot_rms):
    terms = ["total", "KE", "ion-e", "Hartree", "XC", "ion-ion", "TF", "vW", "NL"]
    err = np.abs(et_g - et_o) / nat
    print("\n%s %s per-term |dE|/atom (Ha): %s; potential RMS error %.3e" %
          (name, prec, ", ".join("%s %.2e" % (t, e) for t, e in zip(terms, err)), pot_rms))
    return err


@pytest.mark.parametrize("name", list(CELLS))
def test_headline_eval_fp64(gpu_engine, name):
    c, oc, f, rho, pot_o, et_o, F_o = oracle_case(name)
    s = pcell.setup_slot(gpu_engine, c, native.FP64)
    try:
        # the device-built ion potential and Ewald energy against the oracle's
        assert np.abs(gpu_engine.download(s, 2) - f.ion_pot).max() < 1e-9
        pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho)
        rms = float(np.sqrt(np.mean((pot_g - pot_o) ** 2)))
        err = _report(name, "fp64", c.nion, et_g, et_o, rms)
        assert err.max() < 1e-8
        assert rms < 1e-7
        F_g = gpu_engine.forces(s, c.nion, rho=rho)
        assert np.abs(F_g - F_o).max() < 1e-7
    finally:
        gpu_engine.slot_destroy(s)


@pytest.mark.parametrize("name", list(CELLS))
def test_headline_eval_fp32(gpu_engine, name):
    c, oc, f, rho, pot_o, et_o, _ = oracle_case(name)
    s = pcell.setup_slot(gpu_engine, c, native.FP32)
    try:
        pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho)
        rms = float(np.sqrt(np.mean((pot_g - pot_o) ** 2)))
        err = _report(name, "fp32", c.nion, et_g, et_o, rms)
        assert err.max() * HARTREE_TO_EV < 1e-5
        assert rms < 1e-5
    finally:
        gpu_engine.slot_destroy(s)


def test_headline_cfg2_fp64_solve(gpu_engine):
    """One full FP64 NTN solve of the cfg2 cell to potNorm < 1e-6 against the
    oracle's solve from the same initial density."""
    c, oc, f, _, _, _, _ = oracle_case("cfg2")
    rho0 = wl.initial_density(c, seed=0)
    r_o = ntn.NtnSolver(f, ntn.NtnOptions(conv_check="POT", pot_tol=1e-6)).solve(rho0)
    s = pcell.setup_slot(gpu_engine, c, native.FP64)
    try:
        rho_g, e_g, st = gpu_engine.proj_norm_rho_minimization(
            s, rho0, native.ntn_options(conv_check=native.CONV_POT, pot_tol=1e-6))
        assert st["outcome"] == 0 and r_o.outcome == 0
        err = np.abs(e_g - r_o.energy) / c.nion
        print("\ncfg2 solve: GPU %d evals, oracle %d; max per-term |dE|/atom %.2e Ha" %
              (st["num_evals"], r_o.num_evals, err.max()))
        assert err.max() < 1e-8
        F_g = gpu_engine.forces(s, c.nion)
        F_o, _, _ = ofo.total_forces(oc, r_o.rho)
        assert np.abs(F_g - F_o).max() < 1e-7
    finally:
        gpu_engine.slot_destroy(s)
