"""The cell optimiser (SteepestDecent, Source/CellOptimizers.f90:107-304):
the oracle's restatement against the reference's own cell relaxation of
test/optCell, and the engine's batched driver (relax.CellRelax, device stress
and lattice refresh) against the oracle, for WT and second-order WGC cells."""
import dataclasses

import numpy as np
import pytest

import cases
from oracle import cellopt, ntn
from oracle import functional as fn
from oracle.consts import BOHR, HARTREE_TO_EV
from profess_b200 import recpot, relax, workloads as wl


def test_oracle_cell_relax_follows_the_reference():
    """test/optCell/sampleoutput/displaced.out: the first ten cell steps'
    energies within 2e-5 eV and stresses within 3e-7 Ha/bohr^3 (each density
    solve converges to dE < 1e-6 Ha); the final lattice of displaced.final.geom
    within 5e-4 A.  The last steps, where max|stress| is below 2e-6, follow the
    solves' convergence noise: the reference takes 18 steps, the oracle 14."""
    cell, f, _, c = cases.golden_case("wt_al4_cell")
    ref = c["cell_relax"]
    lat, trace = cellopt.steepest_descent(cell, f.n, ntn.NtnOptions())
    for (e, s, _), r in list(zip(trace, ref["steps"]))[:10]:
        assert abs(e * HARTREE_TO_EV - r["energy_ev"]) < 2e-5
        assert np.abs(s - np.array(r["stress_au"])).max() < 3e-7
    assert np.abs(lat.T * BOHR - np.array(ref["final_lattice_angstrom_rows"])).max() < 5e-4
    assert np.abs(trace[-1][1]).max() < cellopt.TOLS


def check_cell_relax_matches_oracle(eng, max_steps=100):
    cell, f, _, c = cases.golden_case("wt_al4_cell")
    z = np.load(cases.GOLDEN + "/al_hc_recpot.npz")
    sp = recpot.species_from_table(float(z["max_g"]), z["values"], "Al")
    wc = wl.Cell(name="al4_cell", lattice=cell.lattice, frac=cell.frac, species_of_ion=cell.species_of_ion,
                 species=[sp], grid=tuple(f.n))
    run = relax.CellRelax(eng, [wc], max_steps=max_steps)
    try:
        run.run()
        st = run.states[0]
        lat, trace = cellopt.steepest_descent(cell, f.n, ntn.NtnOptions(), max_steps=max_steps)
        assert len(st.history) == len(trace)
        # a lattice step is V dt sigma L^-T with V dt up to ~3e4 bohr^3 a.u.
        # (dt grows 1.2x per step), so stress differences of 1e-12 (FP64
        # rounding of the two sums) reach the lattice as ~2e-8 bohr
        for h, (e, s, L) in zip(st.history, trace):
            assert abs(h["energy"] - e) < 1e-9
            assert np.abs(h["stress"] - s).max() < 1e-10
            assert np.abs(h["lattice"] - L).max() < 1e-7
        assert np.abs(st.cell.lattice - lat).max() < 1e-7
    finally:
        run.close()


def check_wgc_cell_relax_matches_oracle(eng, max_steps=3):
    """A strained second-order WGC Al4 cell: the driver rebuilds the WGC kernel
    at the new N/V after each move and takes WGCStress; three cell steps
    against the oracle's SteepestDecent with the same functional."""
    cell0, f0, _, c = cases.golden_case("wgc_al4_fcc")
    lat = (np.eye(3) + np.diag([0.03, -0.02, 0.01])) @ cell0.lattice
    cell = dataclasses.replace(cell0, lattice=lat)
    z = np.load(cases.GOLDEN + "/al_hc_recpot.npz")
    sp = recpot.species_from_table(float(z["max_g"]), z["values"], "Al")
    wc = wl.Cell(name="al4_wgc", lattice=lat, frac=cell.frac, species_of_ion=cell.species_of_ion, species=[sp],
                 grid=tuple(f0.n), kinetic=5, alpha=c["alpha"], beta=c["beta"], gamma=c["gamma"])
    run = relax.CellRelax(eng, [wc], max_steps=max_steps)
    try:
        run.run()
        st = run.states[0]
        lat_o, trace = cellopt.steepest_descent(cell, f0.n, ntn.NtnOptions(), max_steps=max_steps,
                                                alpha_=c["alpha"], beta_=c["beta"], kinetic=fn.KEDF_WGC,
                                                gamma=c["gamma"])
        assert len(st.history) == len(trace) == max_steps
        assert np.abs(trace[0][1]).max() > 1e-5  # the strain gives a real stress
        for h, (e, s, L) in zip(st.history, trace):
            assert abs(h["energy"] - e) < 1e-9
            assert np.abs(h["stress"] - s).max() < 1e-10
            assert np.abs(h["lattice"] - L).max() < 1e-7
        assert np.abs(st.cell.lattice - lat_o).max() < 1e-7
    finally:
        run.close()


def test_wgc_cell_relax_matches_oracle(emu_engine):
    check_wgc_cell_relax_matches_oracle(emu_engine)


@pytest.mark.gpu
def test_wgc_cell_relax_matches_oracle_on_gpu(gpu_engine):
    check_wgc_cell_relax_matches_oracle(gpu_engine)


def test_cell_relax_matches_oracle(emu_engine):
    check_cell_relax_matches_oracle(emu_engine)


def test_cell_relax_step_cap(emu_engine):
    """max_steps: the cell moves after the last solve, as the reference's loop."""
    check_cell_relax_matches_oracle(emu_engine, max_steps=3)


@pytest.mark.gpu
def test_cell_relax_matches_oracle_on_gpu(gpu_engine):
    check_cell_relax_matches_oracle(gpu_engine)
