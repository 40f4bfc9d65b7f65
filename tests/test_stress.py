"""The engine's stress tensor (ofdft_slot_stress) against the oracle's
CalculateStress restatement on the same density: the optCell Al4 cell (a
sheared lattice, so the off-diagonal and Nyquist terms are exercised) and a
larger synthetic fcc cell; both the given-density and the resident-density
forms, and that the call leaves the slot's solve record as it was; and the
second-order WGC functional's stress on a strained WGC Al4 cell."""
import numpy as np
import pytest

import cases
from oracle import ntn
from oracle import stress as ost
from profess_b200 import cell as pcell
from profess_b200 import native, recpot, workloads as wl


def _golden_slot(eng, prec):
    cell, f, rho_u, c = cases.golden_case("wt_al4_cell")
    z = np.load(cases.GOLDEN + "/al_hc_recpot.npz")
    sp = recpot.species_from_table(float(z["max_g"]), z["values"], "Al")
    wc = wl.Cell(name="al4_cell", lattice=cell.lattice, frac=cell.frac, species_of_ion=cell.species_of_ion,
                 species=[sp], grid=tuple(f.n))
    assert (wc.alpha, wc.beta) == (c["alpha"], c["beta"])
    return cell, f, rho_u, pcell.setup_slot(eng, wc, prec)


def check_stress_matches_oracle(eng, prec=native.FP64, tol=1e-10):
    cell, f, rho_u, s = _golden_slot(eng, prec)
    try:
        r = ntn.NtnSolver(f).solve(rho_u)
        ref = ost.stress(cell, f, r.rho)
        got, parts = eng.stress(s, rho=r.rho, terms=True)
        assert np.abs(got - ref).max() < tol, (got, ref)
        assert np.array_equal(got, got.T)
        assert np.allclose(sum(parts.values()), got, rtol=0, atol=1e-15)
        ew = ost.ewald_stress(cell.lattice, cell.frac, cell.charges())
        assert np.abs(parts["Ewald"] - ew).max() < 1e-12
        assert np.abs(got - eng.stress(s, rho=r.rho, include_ewald=False) - parts["Ewald"]).max() < 1e-15
        # the slot's own solve, then the stress of its resident density
        opts = native.ntn_options(conv_check=native.CONV_POT, pot_tol=1e-7 if prec == native.FP64 else 3e-5,
                                  max_iter=300, stall_line=6)
        eng.start_solve(s, rho_u, opts)
        while eng.run(8):
            pass
        rho_d, e_d, st_d = eng.result(s)
        got2 = eng.stress(s)
        assert np.abs(got2 - ost.stress(cell, f, rho_d)).max() < tol
        rho_d2, e_d2, st_d2 = eng.result(s)
        assert np.array_equal(rho_d, rho_d2) and np.array_equal(e_d, e_d2) and st_d == st_d2
    finally:
        eng.slot_destroy(s)


def check_stress_on_fcc(eng, grid=(48, 48, 48), prec=native.FP64, tol=1e-10):
    c = wl.fcc_al((2, 2, 2), sigma_ang=0.05, grid=grid, seed=5)
    oc, f = cases.workload_functional(c)
    s = pcell.setup_slot(eng, c, prec)
    try:
        rho = cases.random_density(grid, c.num_electrons, c.vol, seed=4, amp=0.2)
        got = eng.stress(s, rho=rho)
        ref = ost.stress(oc, f, rho)
        assert np.abs(got - ref).max() < tol, np.abs(got - ref).max()
    finally:
        eng.slot_destroy(s)


def test_stress_matches_oracle(emu_engine):
    check_stress_matches_oracle(emu_engine)


def test_stress_matches_oracle_fp32_slot(emu_engine):
    """An FP32 slot: the spectra are single precision, the sums FP64."""
    check_stress_matches_oracle(emu_engine, native.FP32, tol=5e-9)


def test_stress_on_fcc(emu_engine):
    check_stress_on_fcc(emu_engine, grid=(24, 24, 24))


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(native.FP64, 1e-10), (native.FP32, 5e-9)])
def test_stress_matches_oracle_on_gpu(gpu_engine, prec, tol):
    check_stress_matches_oracle(gpu_engine, prec, tol)


@pytest.mark.gpu
@pytest.mark.parametrize("grid", [(48, 48, 48), (60, 64, 72)])
def test_stress_on_fcc_on_gpu(gpu_engine, grid):
    check_stress_on_fcc(gpu_engine, grid=grid)


def test_stress_needs_ions(emu_engine):
    c = wl.fcc_al((1, 1, 1), sigma_ang=0.0, grid=(16, 16, 16), seed=0)
    rho = np.full(c.grid, c.num_electrons / c.vol)
    s = pcell._create(emu_engine, c, native.FP64, 0.0)
    try:
        emu_engine.build_wt_kernel(s)
        with pytest.raises(native.OfdftError, match="ion potential"):
            emu_engine.stress(s, rho=rho)
    finally:
        emu_engine.slot_destroy(s)


def check_wgc_stress_matches_oracle(eng, grid=(16, 16, 16), prec=native.FP64, tol=1e-10):
    """The second-order WGC stress (WGCStress) on a strained WGC Al4 cell."""
    cell0, f0, _, c = cases.golden_case("wgc_al4_fcc")
    strain = np.array([[0.02, 0.01, 0.0], [0.01, -0.01, 0.0], [0.0, 0.0, 0.015]])
    lat = (np.eye(3) + strain) @ cell0.lattice
    oc = cases.cs.Cell(lattice=lat, frac=cell0.frac, species_of_ion=cell0.species_of_ion, species=cell0.species)
    f = cases.functional_for(oc, grid, cases.fn.KEDF_WGC, c["alpha"], c["beta"], c["lambda"], c["mu"],
                             c.get("gamma", 2.7))
    z = np.load(cases.GOLDEN + "/al_hc_recpot.npz")
    sp = recpot.species_from_table(float(z["max_g"]), z["values"], "Al")
    wc = wl.Cell(name="wgc", lattice=lat, frac=cell0.frac, species_of_ion=cell0.species_of_ion, species=[sp],
                 grid=tuple(grid), kinetic=native.KEDF_WGC, alpha=c["alpha"], beta=c["beta"],
                 gamma=c.get("gamma", 2.7))
    s = pcell.setup_slot(eng, wc, prec)
    try:
        rho = cases.random_density(grid, oc.num_electrons, oc.vol, seed=9, amp=0.2)
        got, parts = eng.stress(s, rho=rho, terms=True)
        ref = ost.stress(oc, f, rho, gamma=c.get("gamma", 2.7))
        assert np.abs(got - ref).max() < tol, np.abs(got - ref).max()
        assert np.abs(parts["nonlocal"]).max() > 1e-6
    finally:
        eng.slot_destroy(s)


def check_wgc_stress_on_hcp(eng, grid=(16, 16, 24), prec=native.FP64, tol=1e-10):
    """WGC stress on a non-orthogonal (120 degree) hcp Mg cell of the product
    set-up path (Heine-Abarenkov Mg, rho0 = rho* = N/V)."""
    c = wl.hcp_mg((2, 2, 2), sigma_ang=0.05, grid=grid, seed=3)
    assert c.kinetic == native.KEDF_WGC
    oc, f = cases.workload_functional(c)
    s = pcell.setup_slot(eng, c, prec)
    try:
        rho = cases.random_density(grid, c.num_electrons, c.vol, seed=5, amp=0.2)
        got = eng.stress(s, rho=rho)
        ref = ost.stress(oc, f, rho, gamma=c.gamma)
        assert np.abs(got - ref).max() < tol, np.abs(got - ref).max()
        assert abs(got[0, 1]) > 1e-7  # the 120 degree cell has shear terms
    finally:
        eng.slot_destroy(s)


def test_wgc_stress_on_hcp(emu_engine):
    check_wgc_stress_on_hcp(emu_engine)


@pytest.mark.gpu
def test_wgc_stress_on_hcp_on_gpu(gpu_engine):
    check_wgc_stress_on_hcp(gpu_engine, grid=(24, 24, 40))


def test_wgc_stress_matches_oracle(emu_engine):
    check_wgc_stress_matches_oracle(emu_engine)
    check_wgc_stress_matches_oracle(emu_engine, prec=native.FP32, tol=5e-9)


@pytest.mark.gpu
def test_wgc_stress_matches_oracle_on_gpu(gpu_engine):
    check_wgc_stress_matches_oracle(gpu_engine)
    check_wgc_stress_matches_oracle(gpu_engine, grid=(32, 30, 36))
    check_wgc_stress_matches_oracle(gpu_engine, prec=native.FP32, tol=5e-9)
