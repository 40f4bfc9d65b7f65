"""CUDA engine vs the FP64 oracle, through the C ABI.

Tolerances: FP64 potential max relative error 1e-11 and every energy term
within 1e-10 Ha (the contract asks 1e-8 Ha/atom); FP32 slots within 1e-5
relative on the potential and 2e-6 Ha/atom on each energy term."""
import numpy as np
import pytest

import cases
from oracle import functional as fn
from oracle import ntn
from profess_b200 import native

pytestmark = pytest.mark.gpu

GOLDEN = ["wt_al4_displaced", "wgc_al4_fcc"]


@pytest.mark.parametrize("name", GOLDEN)
@pytest.mark.parametrize("opt_sqrt", [True, False])
def test_eval_fp64(gpu_engine, name, opt_sqrt):
    cell, f, _, _ = cases.golden_case(name)
    s = cases.engine_slot(gpu_engine, f, cell)
    try:
        for seed in (1, 2):
            rho = cases.random_density(f.n, cell.num_electrons, cell.vol, seed=seed)
            pot_o, et_o = fn.calculate_potential_plus(f, rho, opt_sqrt=opt_sqrt)
            pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho, opt_sqrt=opt_sqrt)
            assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < 1e-11
            assert np.abs(et_g - et_o).max() < 1e-10
    finally:
        gpu_engine.slot_destroy(s)


@pytest.mark.parametrize("name", GOLDEN)
def test_eval_fp32(gpu_engine, name):
    cell, f, _, _ = cases.golden_case(name)
    s = cases.engine_slot(gpu_engine, f, cell, precision=1)
    try:
        rho = cases.random_density(f.n, cell.num_electrons, cell.vol, seed=3)
        pot_o, et_o = fn.calculate_potential_plus(f, rho)
        pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho)
        assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < 1e-5
        nat = len(cell.frac)
        assert np.abs(et_g - et_o).max() / nat < 2e-6
    finally:
        gpu_engine.slot_destroy(s)


@pytest.mark.parametrize("n", [(16, 18, 20), (15, 21, 14), (25, 12, 27), (7, 10, 9), (32, 30, 28)])
def test_eval_odd_and_mixed_radix_grids(gpu_engine, n):
    cell, _, _, _ = cases.golden_case("wt_al4_displaced")
    f = cases.functional_for(cell, n, fn.KEDF_WT, 5 / 6, 5 / 6)
    s = cases.engine_slot(gpu_engine, f, cell)
    try:
        rho = cases.random_density(n, cell.num_electrons, cell.vol, seed=4)
        pot_o, et_o = fn.calculate_potential_plus(f, rho)
        pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho)
        assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < 1e-11
        assert np.abs(et_g - et_o).max() < 1e-10
    finally:
        gpu_engine.slot_destroy(s)


@pytest.mark.parametrize("n", [(32, 48, 96), (96, 12, 10), (10, 72, 120), (9, 64, 80)])
def test_eval_two_step_lengths(gpu_engine, n):
    """Lengths with the two-step register transform along x, y and z."""
    cell, _, _, _ = cases.golden_case("wt_al4_displaced")
    f = cases.functional_for(cell, n, fn.KEDF_WT, 5 / 6, 5 / 6)
    s = cases.engine_slot(gpu_engine, f, cell)
    try:
        rho = cases.random_density(n, cell.num_electrons, cell.vol, seed=5)
        pot_o, et_o = fn.calculate_potential_plus(f, rho)
        pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho)
        assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < 1e-11
        assert np.abs(et_g - et_o).max() < 1e-10
    finally:
        gpu_engine.slot_destroy(s)


@pytest.mark.parametrize("n", [(8, 128, 160), (6, 256, 192), (160, 6, 5)])
def test_eval_two_step_lengths_fp32(gpu_engine, n):
    """FP32 two-step lengths with a 16-point second step (WGC).  FP32 gives a
    max-relative potential error of up to ~5e-4 on these random densities
    with either transform, hence 1e-3 (energies per term to 5e-5 Ha)."""
    cell, _, _, _ = cases.golden_case("wgc_al4_fcc")
    f = cases.functional_for(cell, n, fn.KEDF_WGC, 1.2060113295832982827, 0.46065533708336838393)
    s = cases.engine_slot(gpu_engine, f, cell, precision=native.FP32)
    try:
        rho = cases.random_density(n, cell.num_electrons, cell.vol, seed=6)
        pot_o, et_o = fn.calculate_potential_plus(f, rho)
        pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho)
        assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < 1e-3
        assert np.abs(et_g - et_o).max() < 5e-5
    finally:
        gpu_engine.slot_destroy(s)


@pytest.mark.parametrize("name", GOLDEN)
def test_solve_fp64_matches_oracle_trajectory(gpu_engine, name):
    cell, f, rho_u, _ = cases.golden_case(name)
    s = cases.engine_slot(gpu_engine, f, cell)
    try:
        r_o = ntn.NtnSolver(f).solve(rho_u)
        rho_g, e_g, st = gpu_engine.proj_norm_rho_minimization(s, rho_u)
        hist = gpu_engine.history(s)
        assert st["outcome"] == r_o.outcome == 0
        assert st["num_evals"] == r_o.num_evals
        assert [h["ncg"] for h in hist] == [h["ncg"] for h in r_o.history]
        assert np.abs(e_g - r_o.energy).max() < 1e-9
        assert np.abs(rho_g - r_o.rho).max() < 1e-9
    finally:
        gpu_engine.slot_destroy(s)
