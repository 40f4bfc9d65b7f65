"""CUDA engine features against the oracle (GPU): device set-up of kernels
and ion potential, spline forces, large FFT plans, the product set-up path on
a synthetic workload cell, mixed precision, batch invariance (one precision,
and both precisions in concurrent graph branches), serving."""
import numpy as np
import pytest

import cases
from oracle import cellsetup as cs
from oracle import forces as ofo
from oracle import functional as fn
from oracle import kedf_kernels as kk
from oracle import ntn
from oracle.consts import HARTREE_TO_EV
from profess_b200 import cell as pcell
from profess_b200 import native, serving, workloads as wl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["wt_al4_displaced", "wgc_al4_fcc"])
def test_device_setup_and_forces(gpu_engine, name):
    cell, f, _, _ = cases.golden_case(name)
    rho0 = cell.num_electrons / cell.vol
    s = gpu_engine.slot_create(f.n, cell.lattice, kinetic=f.kinetic, alpha=f.alpha, beta=f.beta, rho0=rho0,
                               rho_s=f.rho_s, ion_ion=f.ion_ion)
    try:
        if f.kinetic == fn.KEDF_WT:
            gpu_engine.build_wt_kernel(s)
        else:
            gpu_engine.build_wgc_kernel(s, kk.wgc_radial_tables(f.alpha, f.beta, 2.7))
        gpu_engine.build_ion_potential(s, cell.frac, cell.species_of_ion, cell.species)
        assert np.abs(gpu_engine.download(s, 2) - f.ion_pot).max() < 1e-12
        rho = cases.random_density(f.n, cell.num_electrons, cell.vol, seed=4)
        pot_o, et_o = fn.calculate_potential_plus(f, rho)
        pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho)
        assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < 1e-11
        assert np.abs(et_g - et_o).max() < 1e-10
        F = gpu_engine.forces(s, len(cell.frac), rho=rho)
        Fo, _, _ = ofo.total_forces(cell, rho)
        assert np.abs(F - Fo).max() < 1e-10
    finally:
        gpu_engine.slot_destroy(s)


@pytest.mark.parametrize("n", [(16, 20, 256), (160, 12, 10), (7, 250, 9), (27, 25, 49)])
def test_large_and_odd_plans(gpu_engine, n):
    cell, _, _, _ = cases.golden_case("wt_al4_displaced")
    f = cases.functional_for(cell, n, fn.KEDF_WT, 5 / 6, 5 / 6)
    s = cases.engine_slot(gpu_engine, f, cell)
    try:
        rho = cases.random_density(n, cell.num_electrons, cell.vol, seed=6)
        pot_o, et_o = fn.calculate_potential_plus(f, rho)
        pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho)
        assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < 1e-11
        assert np.abs(et_g - et_o).max() < 1e-10
    finally:
        gpu_engine.slot_destroy(s)


def test_wgc_hcp_cell(gpu_engine):
    """WGC on a non-orthogonal (120 degree) hcp Mg cell."""
    c = wl.hcp_mg((2, 2, 2), sigma_ang=0.05, grid=(24, 24, 40), seed=3)
    mx, vals = wl.heine_abarenkov_table(2.0, 1.3, 0.1)
    ocell = cs.Cell(lattice=c.lattice, frac=c.frac, species_of_ion=c.species_of_ion,
                    species=[cs.species_from_table(mx, vals, "Mg")])
    f = cases.functional_for(ocell, c.grid, fn.KEDF_WGC, c.alpha, c.beta)
    s = cases.engine_slot(gpu_engine, f, ocell)
    try:
        rho = cases.random_density(c.grid, ocell.num_electrons, ocell.vol, seed=7)
        pot_o, et_o = fn.calculate_potential_plus(f, rho)
        pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho)
        assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < 1e-11
        assert np.abs(et_g - et_o).max() < 1e-10
    finally:
        gpu_engine.slot_destroy(s)


def test_workload_cfg1_solve(gpu_engine):
    """Product set-up path (device kernels, device ion potential, host Ewald) and
    an FP64 NTN solve to potNorm < 1e-6, against the oracle.  The device spreads
    the ion structure factor with atomic adds, so its ion potential differs from
    the oracle's in the last bits and the energies agree to 1e-8 Ha, not 1e-10."""
    c = wl.config_cell(1)
    mx, vals = wl.heine_abarenkov_table(3.0, 1.15, 0.1)
    ocell = cs.Cell(lattice=c.lattice, frac=c.frac, species_of_ion=c.species_of_ion,
                    species=[cs.species_from_table(mx, vals, "Al")])
    f = cases.functional_for(ocell, c.grid, fn.KEDF_WT, 5 / 6, 5 / 6)
    s = pcell.setup_slot(gpu_engine, c)
    try:
        rho0 = wl.initial_density(c)
        r_o = ntn.NtnSolver(f, ntn.NtnOptions(conv_check="POT", pot_tol=1e-6)).solve(rho0)
        _, e_g, st = gpu_engine.proj_norm_rho_minimization(
            s, rho0, native.ntn_options(conv_check=native.CONV_POT, pot_tol=1e-6))
        assert st["outcome"] == 0 and abs(st["num_evals"] - r_o.num_evals) <= 2
        assert np.abs(e_g - r_o.energy).max() < 1e-8
    finally:
        gpu_engine.slot_destroy(s)


def test_mixed_precision_energy_error(gpu_engine):
    c = wl.fcc_al((2, 2, 2), sigma_ang=0.05, grid=(48, 48, 48), seed=2)
    e_ii = pcell.ion_ion_energy(gpu_engine.lib, c)
    s32 = pcell.setup_slot(gpu_engine, c, native.FP32, ion_ion=e_ii)
    s64 = pcell.setup_slot(gpu_engine, c, native.FP64, ion_ion=e_ii)
    try:
        rho0 = wl.initial_density(c)
        _, e_ref, _ = gpu_engine.proj_norm_rho_minimization(
            s64, rho0, native.ntn_options(conv_check=native.CONV_POT, pot_tol=1e-7))
        gpu_engine.start_solve(s32, rho0, native.ntn_options(conv_check=native.CONV_POT, pot_tol=1e-5,
                                                            stall_line=6))
        while gpu_engine.run(8):
            pass
        gpu_engine.start_solve_from_slot(s64, s32, native.ntn_options(conv_check=native.CONV_POT,
                                                                      pot_tol=1e-7, max_iter=2))
        while gpu_engine.run(8):
            pass
        _, e_mix, st = gpu_engine.result(s64, want_rho=False)
        assert abs(e_mix[0] - e_ref[0]) * HARTREE_TO_EV / c.nion < 1e-5
        assert st["iterations"] <= 2
    finally:
        gpu_engine.slot_destroy(s32)
        gpu_engine.slot_destroy(s64)


def test_batch_invariance_on_gpu(gpu_engine):
    """Each solve gives the same result alone and batched with others."""
    cells = [wl.fcc_al((1, 1, 1), sigma_ang=0.05, grid=(24, 24, 24), seed=i) for i in range(3)]
    cells.append(wl.fcc_al((2, 1, 1), sigma_ang=0.05, grid=(40, 20, 20), seed=9))
    slots = [pcell.setup_slot(gpu_engine, c) for c in cells]
    try:
        rho = [wl.initial_density(c, seed=i) for i, c in enumerate(cells)]
        alone = [gpu_engine.proj_norm_rho_minimization(s, r) for s, r in zip(slots, rho)]
        for s, r in zip(slots, rho):
            gpu_engine.start_solve(s, r)
        while gpu_engine.run(8):
            pass
        for s, a in zip(slots, alone):
            rb, eb, stb = gpu_engine.result(s)
            assert np.array_equal(eb, a[1]) and np.array_equal(rb, a[0])
            assert stb["num_evals"] == a[2]["num_evals"]
    finally:
        for s in slots:
            gpu_engine.slot_destroy(s)


def test_two_precisions_in_one_graph_match_alone(gpu_engine):
    """FP64 and FP32 slots running together take two concurrent branches of
    the engine's graphs; each solve must give bit for bit what it gives with
    its precision running alone (one branch).  One FP32 cell is WGC (split y/z
    path), the others WT (fused y-z pass)."""
    cells = [wl.fcc_al((1, 1, 1), sigma_ang=0.05, grid=(24, 24, 24), seed=i) for i in range(3)]
    cells.append(wl.fcc_al((1, 1, 2), sigma_ang=0.05, grid=(24, 24, 48), seed=7, kinetic=5))
    cells[-1].alpha, cells[-1].beta = (5 + 5 ** 0.5) / 6, (5 - 5 ** 0.5) / 6
    precs = [native.FP64, native.FP32, native.FP64, native.FP32]
    o64 = native.ntn_options(conv_check=native.CONV_POT, pot_tol=1e-6, max_iter=300)
    o32 = native.ntn_options(conv_check=native.CONV_POT, pot_tol=3e-5, max_iter=300, stall_line=6)
    opts = [o64 if p == native.FP64 else o32 for p in precs]
    slots = [pcell.setup_slot(gpu_engine, c, p) for c, p in zip(cells, precs)]
    try:
        rho = [wl.initial_density(c, seed=i) for i, c in enumerate(cells)]
        alone = [gpu_engine.proj_norm_rho_minimization(s, r, o) for s, r, o in zip(slots, rho, opts)]
        for s, r, o in zip(slots, rho, opts):
            gpu_engine.start_solve(s, r, o)
        while gpu_engine.run(8):
            pass
        for s, a in zip(slots, alone):
            rb, eb, stb = gpu_engine.result(s)
            assert np.array_equal(eb, a[1]) and np.array_equal(rb, a[0])
            assert stb["num_evals"] == a[2]["num_evals"] and stb["outcome"] == a[2]["outcome"]
    finally:
        for s in slots:
            gpu_engine.slot_destroy(s)


def test_serving_results_same_alone_and_in_the_mix(gpu_engine):
    rng = np.random.default_rng(5)
    reqs = []
    for i in range(4):
        c = wl.fcc_al((1, 1, 1 + i % 2), sigma_ang=0.05, grid=(24, 24, 24 * (1 + i % 2)), seed=i,
                      kinetic=4 if i != 3 else 5)
        if c.kinetic == 5:
            c.alpha, c.beta = (5 + 5 ** 0.5) / 6, (5 - 5 ** 0.5) / 6
        reqs.append(serving.Request(rid=i, cell=c, arrival=float(rng.uniform(0, 0.01)), seed=i,
                                    mode=serving.MODE_MIXED if i % 2 == 0 else serving.MODE_FP64))

    def run(rs):
        srv = serving.Server(gpu_engine, hbm_budget=8 << 30, ticks_per_poll=4)
        for r in rs:
            srv.submit(r)
        return {r.rid: r for r in srv.run_until_done(timeout=600)}

    mix = run(reqs)
    for r in reqs:
        a = run([r])[r.rid]
        assert np.array_equal(a.energy, mix[r.rid].energy)


@pytest.mark.parametrize("n,kinetic,prec", [((512, 6, 4), fn.KEDF_WT, native.FP64),
                                             ((4, 512, 6), fn.KEDF_WGC, native.FP64),
                                             ((6, 4, 512), fn.KEDF_WGC, native.FP64),
                                             ((8, 6, 512), fn.KEDF_WT, native.FP32)])
def test_maximum_lengths(gpu_engine, n, kinetic, prec):
    """512, the longest length a slot takes, along each axis (largest shared-memory
    tiles).  A 512-point axis over this cell's 7.6 bohr gives large |G|^2 kernel
    factors, so the potential is ill-conditioned in the density: rounding the
    density to FP32 alone moves the oracle's WGC potential by 3.7e-3 (relative to
    its maximum).  The host-emulated kernels give 4e-11 in FP64 (WGC) and 1.3e-3
    in FP32 (WT), hence 1e-10 and 5e-3."""
    cell, _, _, _ = cases.golden_case("wgc_al4_fcc")
    ab = (5 / 6, 5 / 6) if kinetic == fn.KEDF_WT else (1.2060113295832982827, 0.46065533708336838393)
    f = cases.functional_for(cell, n, kinetic, *ab)
    s = cases.engine_slot(gpu_engine, f, cell, precision=prec)
    try:
        rho = cases.random_density(n, cell.num_electrons, cell.vol, seed=8)
        pot_o, et_o = fn.calculate_potential_plus(f, rho)
        pot_g, et_g = gpu_engine.calculate_potential_plus(s, rho)
        tol_pot, tol_e = (1e-10, 1e-10) if prec == native.FP64 else (5e-3, 5e-5)
        assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < tol_pot
        assert np.abs(et_g - et_o).max() < tol_e
    finally:
        gpu_engine.slot_destroy(s)


def test_cancel_and_tick_budget_on_gpu(gpu_engine):
    """A solve cut off by its tick budget, or cancelled while running, leaves the
    slot idle; the next solve on it matches a fresh one."""
    cell, f, rho_u, _ = cases.golden_case("wt_al4_displaced")
    s = cases.engine_slot(gpu_engine, f, cell)
    try:
        with pytest.raises(native.OfdftError) as ei:
            gpu_engine.proj_norm_rho_minimization(s, rho_u, native.ntn_options(max_ticks=3))
        assert ei.value.code == 8 and gpu_engine.poll(s)
        gpu_engine.start_solve(s, rho_u)
        gpu_engine.run(2)
        gpu_engine.cancel(s)
        assert gpu_engine.poll(s)
        r_o = ntn.NtnSolver(f).solve(rho_u)
        _, e_g, st = gpu_engine.proj_norm_rho_minimization(s, rho_u)
        assert st["num_evals"] == r_o.num_evals and abs(e_g[0] - r_o.energy[0]) < 1e-9
    finally:
        gpu_engine.slot_destroy(s)


def test_device_ewald_on_gpu(gpu_engine):
    from test_emu_engine import check_device_ewald
    check_device_ewald(gpu_engine)


def test_repeated_ion_builds_hold_device_memory(gpu_engine):
    """A geometry loop's ion-potential rebuilds reuse the slot's table buffer:
    the device's free memory does not shrink over 40 rebuilds."""
    import torch
    c = wl.fcc_al((2, 2, 2), sigma_ang=0.05, grid=(48, 48, 48), seed=3)
    s = pcell.setup_slot(gpu_engine, c)
    try:
        gpu_engine.build_ion_potential(s, c.frac, c.species_of_ion, c.species)
        free0, _ = torch.cuda.mem_get_info()
        rng = np.random.default_rng(0)
        for _ in range(40):
            fr = np.mod(c.frac + rng.normal(0, 1e-3, c.frac.shape), 1.0)
            gpu_engine.build_ion_potential(s, fr, c.species_of_ion, c.species)
        free1, _ = torch.cuda.mem_get_info()
        assert free0 - free1 < 2 << 20
    finally:
        gpu_engine.slot_destroy(s)


def test_copy_tables_on_gpu(gpu_engine):
    from test_emu_engine import check_copy_tables
    check_copy_tables(gpu_engine)


@pytest.mark.parametrize("n,prec", [((8, 9, 10), native.FP64), ((6, 14, 9), native.FP64), ((5, 25, 8), native.FP64),
                                    ((4, 49, 6), native.FP64), ((6, 16, 15), native.FP64), ((5, 18, 12), native.FP64),
                                    ((4, 10, 14), native.FP64), ((4, 12, 7), native.FP64), ((6, 16, 10), native.FP32),
                                    ((5, 32, 9), native.FP32), ((4, 15, 16), native.FP32)])
def test_wgc_fused_yz_radices_on_gpu(gpu_engine, n, prec):
    """WGC groups in the fused y-z pass with the WGC operator in a last y
    stage of radix 2 to 16, against the oracle (the grids of the emulated
    test_eval_wgc_fused_yz_* cases)."""
    from test_emu_engine import WGC_AB, _eval_parity
    cell, _, _, _ = cases.golden_case("wgc_al4_fcc")
    f = cases.functional_for(cell, n, fn.KEDF_WGC, *WGC_AB)
    if prec == native.FP64:
        _eval_parity(gpu_engine, f, cell, seed=7)
    else:
        _eval_parity(gpu_engine, f, cell, seed=8, prec=native.FP32, tol_pot=1e-5, tol_e=2e-5)

