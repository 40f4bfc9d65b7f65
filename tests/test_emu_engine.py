"""The engine's kernel logic, run by the host-emulation build, against the oracle (CPU).

tests/_emu/libprofess_b200_emu.so compiles the same block functions as the
CUDA library for the host and runs every block with one thread.  These tests
check the pass logic (FFT passes, field tables, k-space operators, epilogue,
reductions, NTN controller, set-up passes) against the FP64 oracle at the
tolerances the GPU tests use.  The GPU tests (test_gpu_*.py) repeat the
parity checks on the CUDA build."""
import numpy as np
import pytest

import cases
from oracle import forces as ofo
from oracle import functional as fn
from oracle import kedf_kernels as kk
from oracle import ntn
from profess_b200 import native


def _eval_parity(eng, f, cell, seed=1, opt_sqrt=True, prec=native.FP64, tol_pot=1e-11, tol_e=1e-10):
    s = cases.engine_slot(eng, f, cell, precision=prec)
    try:
        rho = cases.random_density(f.n, cell.num_electrons, cell.vol, seed=seed)
        pot_o, et_o = fn.calculate_potential_plus(f, rho, opt_sqrt=opt_sqrt)
        pot_g, et_g = eng.calculate_potential_plus(s, rho, opt_sqrt=opt_sqrt)
        assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < tol_pot
        assert np.abs(et_g - et_o).max() < tol_e
    finally:
        eng.slot_destroy(s)


@pytest.mark.parametrize("name", ["wt_al4_displaced", "wgc_al4_fcc"])
@pytest.mark.parametrize("opt_sqrt", [True, False])
def test_eval_golden_cells(emu_engine, name, opt_sqrt):
    cell, f, _, _ = cases.golden_case(name)
    _eval_parity(emu_engine, f, cell, opt_sqrt=opt_sqrt)


@pytest.mark.parametrize("n", [(16, 18, 20), (15, 21, 14), (25, 12, 27), (7, 10, 9), (8, 14, 49), (2, 3, 5)])
def test_eval_mixed_radix_and_odd_grids(emu_engine, n):
    cell, _, _, _ = cases.golden_case("wt_al4_displaced")  # non-orthogonal lattice
    f = cases.functional_for(cell, n, fn.KEDF_WT, 5 / 6, 5 / 6)
    _eval_parity(emu_engine, f, cell, seed=2)


@pytest.mark.parametrize("n", [(32, 48, 96), (10, 72, 120), (9, 64, 80), (96, 12, 10), (120, 9, 8)])
def test_eval_two_step_lengths(emu_engine, n):
    """Lengths with the two-step register transform (R1 x R2) along x, y, z."""
    cell, _, _, _ = cases.golden_case("wt_al4_displaced")
    f = cases.functional_for(cell, n, fn.KEDF_WT, 5 / 6, 5 / 6)
    _eval_parity(emu_engine, f, cell, seed=5)


@pytest.mark.parametrize("n", [(8, 128, 160), (6, 256, 192), (5, 240, 144), (160, 6, 5), (256, 4, 6)])
def test_eval_two_step_lengths_fp32(emu_engine, n):
    """FP32 two-step lengths with a 16-point second step.  On these random
    WGC densities FP32 gives a max-relative potential error of 1.6e-4 to
    5.3e-4 whatever the transform: the generic Stockham lengths next to these
    show the same (126 x 162: 1.59e-4 vs 128 x 160: 1.58e-4; 252 x 196:
    5.03e-4 vs 256 x 192: 5.28e-4), hence 1e-3."""
    cell, _, _, _ = cases.golden_case("wgc_al4_fcc")
    f = cases.functional_for(cell, n, fn.KEDF_WGC, 1.2060113295832982827, 0.46065533708336838393)
    _eval_parity(emu_engine, f, cell, seed=6, prec=native.FP32, tol_pot=1e-3, tol_e=5e-5)


WGC_AB = (1.2060113295832982827, 0.46065533708336838393)


@pytest.mark.parametrize("n", [(8, 9, 10), (6, 14, 9), (5, 25, 8), (4, 49, 6), (6, 16, 15), (5, 18, 12),
                               (4, 10, 14), (4, 12, 7)])
def test_eval_wgc_fused_yz_radices(emu_engine, n):
    """WGC groups in the fused y-z pass (three planes a task): y lengths whose
    last stage, where the WGC operator sits, has radix 9, 2, 5, 7, 4, 3, 10 and
    12, against the oracle in FP64."""
    cell, _, _, _ = cases.golden_case("wgc_al4_fcc")
    f = cases.functional_for(cell, n, fn.KEDF_WGC, *WGC_AB)
    _eval_parity(emu_engine, f, cell, seed=7)


@pytest.mark.parametrize("n", [(6, 16, 10), (5, 32, 9), (4, 15, 16)])
def test_eval_wgc_fused_yz_fp32(emu_engine, n):
    """The same in FP32 (radix 16, 4 and 15 in the operator stage)."""
    cell, _, _, _ = cases.golden_case("wgc_al4_fcc")
    f = cases.functional_for(cell, n, fn.KEDF_WGC, *WGC_AB)
    _eval_parity(emu_engine, f, cell, seed=8, prec=native.FP32, tol_pot=1e-5, tol_e=2e-5)


def test_eval_wt_alpha_ne_beta(emu_engine):
    cell, _, _, _ = cases.golden_case("wt_al4_displaced")
    f = cases.functional_for(cell, (16, 16, 18), fn.KEDF_WT, 1.0, 2.0 / 3.0)
    _eval_parity(emu_engine, f, cell, seed=3)


def test_eval_fp32(emu_engine):
    cell, f, _, _ = cases.golden_case("wgc_al4_fcc")
    _eval_parity(emu_engine, f, cell, prec=native.FP32, tol_pot=1e-5, tol_e=2e-5)


@pytest.mark.parametrize("name", ["wt_al4_displaced", "wgc_al4_fcc"])
def test_solve_trajectory(emu_engine, name):
    cell, f, rho_u, _ = cases.golden_case(name)
    s = cases.engine_slot(emu_engine, f, cell)
    try:
        r_o = ntn.NtnSolver(f).solve(rho_u)
        rho_g, e_g, st = emu_engine.proj_norm_rho_minimization(s, rho_u)
        hist = emu_engine.history(s)
        assert st["outcome"] == r_o.outcome == 0
        assert st["num_evals"] == r_o.num_evals
        assert [h["ncg"] for h in hist] == [h["ncg"] for h in r_o.history]
        assert [h["nline"] for h in hist] == [h["nline"] for h in r_o.history]
        assert np.abs(e_g - r_o.energy).max() < 1e-9
        assert np.abs(rho_g - r_o.rho).max() < 1e-9
    finally:
        emu_engine.slot_destroy(s)


def test_solve_pot_convergence_option(emu_engine):
    cell, f, rho_u, _ = cases.golden_case("wt_al4_cell")
    s = cases.engine_slot(emu_engine, f, cell)
    try:
        r_o = ntn.NtnSolver(f, ntn.NtnOptions(conv_check="POT", pot_tol=1e-7)).solve(rho_u)
        _, e_g, st = emu_engine.proj_norm_rho_minimization(
            s, rho_u, native.ntn_options(conv_check=native.CONV_POT, pot_tol=1e-7))
        assert st["iterations"] == r_o.iterations and st["pot_norm"] < 1e-7
        assert abs(e_g[0] - r_o.energy[0]) < 1e-10
    finally:
        emu_engine.slot_destroy(s)


def test_batched_slots_match_single(emu_engine):
    """Two different cells solved together give the same result as each alone."""
    cell_a, f_a, rho_a, _ = cases.golden_case("wt_al4_displaced")
    cell_b, f_b, rho_b, _ = cases.golden_case("wgc_al4_fcc")
    sa = cases.engine_slot(emu_engine, f_a, cell_a)
    sb = cases.engine_slot(emu_engine, f_b, cell_b)
    try:
        alone_a = emu_engine.proj_norm_rho_minimization(sa, rho_a)
        alone_b = emu_engine.proj_norm_rho_minimization(sb, rho_b)
        emu_engine.start_solve(sa, rho_a)
        emu_engine.start_solve(sb, rho_b)
        while emu_engine.run(8):
            pass
        ra, ea, _ = emu_engine.result(sa)
        rb, eb, _ = emu_engine.result(sb)
        assert np.array_equal(ea, alone_a[1]) and np.array_equal(ra, alone_a[0])
        assert np.array_equal(eb, alone_b[1]) and np.array_equal(rb, alone_b[0])
    finally:
        emu_engine.slot_destroy(sa)
        emu_engine.slot_destroy(sb)


@pytest.mark.parametrize("name", ["wt_al4_displaced", "wgc_al4_fcc"])
def test_device_setup_matches_oracle(emu_engine, name):
    """WT/WGC kernels and the B-spline ion potential built by the library."""
    cell, f, _, _ = cases.golden_case(name)
    lib = emu_engine.lib
    rho0 = cell.num_electrons / cell.vol
    s = emu_engine.slot_create(f.n, cell.lattice, kinetic=f.kinetic, alpha=f.alpha, beta=f.beta, rho0=rho0,
                               rho_s=f.rho_s, ion_ion=f.ion_ion)
    try:
        if f.kinetic == fn.KEDF_WT:
            emu_engine.build_wt_kernel(s)
        else:
            tabs = native.wgc_radial_tables(lib, f.alpha, f.beta, 2.7)
            ref = kk.wgc_radial_tables(f.alpha, f.beta, 2.7)
            for a, b in zip(tabs, ref):
                assert np.abs(a - b).max() <= 1e-5 * (1 + np.abs(b).max())
            emu_engine.build_wgc_kernel(s, ref)  # same tables as the oracle: exact parity below
        emu_engine.build_ion_potential(s, cell.frac, cell.species_of_ion, cell.species)
        v = emu_engine.download(s, 2)
        assert np.abs(v - f.ion_pot).max() < 1e-12
        rho = cases.random_density(f.n, cell.num_electrons, cell.vol, seed=4)
        pot_o, et_o = fn.calculate_potential_plus(f, rho)
        pot_g, et_g = emu_engine.calculate_potential_plus(s, rho)
        assert np.abs(pot_g - pot_o).max() / np.abs(pot_o).max() < 1e-11
        assert np.abs(et_g - et_o).max() < 1e-10
        F = emu_engine.forces(s, len(cell.frac), rho=rho)
        Fo, _, _ = ofo.total_forces(cell, rho)
        assert np.abs(F - Fo).max() < 1e-10
    finally:
        emu_engine.slot_destroy(s)


def test_mixed_precision_refinement(emu_engine):
    """FP32 solve to its floor, FP64 refinement from the device-resident result."""
    cell, f, rho_u, _ = cases.golden_case("wt_al4_displaced")
    s32 = cases.engine_slot(emu_engine, f, cell, precision=native.FP32)
    s64 = cases.engine_slot(emu_engine, f, cell, precision=native.FP64)
    try:
        ref = ntn.NtnSolver(f, ntn.NtnOptions(conv_check="POT", pot_tol=1e-7)).solve(rho_u)
        emu_engine.start_solve(s32, rho_u, native.ntn_options(conv_check=native.CONV_POT, pot_tol=1e-6,
                                                              stall_line=6))
        while emu_engine.run(8):
            pass
        _, e32, st32 = emu_engine.result(s32, want_rho=False)
        emu_engine.start_solve_from_slot(s64, s32, native.ntn_options(conv_check=native.CONV_POT,
                                                                      pot_tol=1e-7, max_iter=3))
        while emu_engine.run(8):
            pass
        _, e64, st64 = emu_engine.result(s64, want_rho=False)
        nat = len(cell.frac)
        ev = 27.2113834
        assert abs(e64[0] - ref.energy[0]) * ev / nat < 1e-5
        assert st32["num_evals"] > 0 and st64["iterations"] <= 3
    finally:
        emu_engine.slot_destroy(s32)
        emu_engine.slot_destroy(s64)


def test_nan_density_reports_status(emu_engine):
    cell, f, _, _ = cases.golden_case("wt_al4_displaced")
    s = cases.engine_slot(emu_engine, f, cell)
    try:
        rho = cases.random_density(f.n, cell.num_electrons, cell.vol, seed=1)
        rho[3, 4, 5] = np.nan
        with pytest.raises(native.OfdftError) as ei:
            emu_engine.calculate_potential_plus(s, rho)
        assert ei.value.code == 5
    finally:
        emu_engine.slot_destroy(s)


def test_invalid_slot_arguments(emu_engine):
    cell, f, _, _ = cases.golden_case("wt_al4_displaced")
    with pytest.raises(native.OfdftError) as ei:
        emu_engine.slot_create((16, 16, 11), cell.lattice)  # 11 is not 7-smooth
    assert ei.value.code == 1
    s = cases.engine_slot(emu_engine, f, cell)
    try:
        with pytest.raises(native.OfdftError):
            emu_engine.set_kernel(s, np.zeros((4,) + f.kernel.shape[1:]))  # WT takes one plane
    finally:
        emu_engine.slot_destroy(s)


def test_tick_budget_timeout_leaves_the_slot_usable(emu_engine):
    """A blocking solve that runs out of ticks returns OFDFT_ETIMEOUT and stops
    the slot, which then solves normally."""
    cell, f, rho_u, _ = cases.golden_case("wt_al4_displaced")
    s = cases.engine_slot(emu_engine, f, cell)
    try:
        with pytest.raises(native.OfdftError) as ei:
            emu_engine.proj_norm_rho_minimization(s, rho_u, native.ntn_options(max_ticks=3))
        assert ei.value.code == 8
        assert emu_engine.poll(s)
        r_o = ntn.NtnSolver(f).solve(rho_u)
        _, e_g, st = emu_engine.proj_norm_rho_minimization(s, rho_u)
        assert st["num_evals"] == r_o.num_evals and abs(e_g[0] - r_o.energy[0]) < 1e-9
    finally:
        emu_engine.slot_destroy(s)


def test_cancel_a_running_solve(emu_engine):
    cell, f, rho_u, _ = cases.golden_case("wt_al4_displaced")
    s = cases.engine_slot(emu_engine, f, cell)
    try:
        emu_engine.start_solve(s, rho_u)
        emu_engine.run(2)
        assert not emu_engine.poll(s)
        emu_engine.cancel(s)
        assert emu_engine.poll(s)
        assert emu_engine.run(4) == 0  # nothing left running
    finally:
        emu_engine.slot_destroy(s)


def test_engine_slot_capacity():
    """The 257th slot of an engine is refused with OFDFT_ENOMEM; freed slots are reused."""
    from profess_b200 import build
    eng = native.Engine(build.build_emu())  # an engine of its own: it fills every slot
    cell, _, _, _ = cases.golden_case("wt_al4_displaced")
    slots = []
    try:
        for _ in range(256):
            slots.append(eng.slot_create((2, 3, 5), cell.lattice))
        with pytest.raises(native.OfdftError) as ei:
            eng.slot_create((2, 3, 5), cell.lattice)
        assert ei.value.code == 3
        eng.slot_destroy(slots.pop())
        slots.append(eng.slot_create((2, 3, 5), cell.lattice))
    finally:
        for s in slots:
            eng.slot_destroy(s)
        eng.close()


def check_device_ewald(eng):
    """The engine's device Ewald sum (energy into the slot's table, forces) against the oracle."""
    from oracle import ewald as oew
    from profess_b200 import cell as pcell, workloads as wl
    for c in (wl.fcc_al((2, 1, 1), sigma_ang=0.1, grid=(16, 8, 8), seed=5),
              wl.hcp_mg((2, 1, 1), sigma_ang=0.05, grid=(12, 6, 10), seed=2)):
        s = pcell.setup_slot(eng, c)
        try:
            e, f = eng.ewald(s, c.nion)
            eo, fo = oew.ewald(c.lattice, c.frac, c.charges(), True)
            assert abs(e - eo) < 1e-10 * max(1.0, abs(eo)) and np.abs(f - fo).max() < 1e-10
            F = eng.forces(s, c.nion, rho=cases.random_density(c.grid, c.num_electrons, c.vol, seed=1))
            F0 = eng.forces(s, c.nion, rho=cases.random_density(c.grid, c.num_electrons, c.vol, seed=1),
                            include_ewald=False)
            assert np.abs((F - F0) - fo).max() < 1e-10
        finally:
            eng.slot_destroy(s)


def test_device_ewald(emu_engine):
    check_device_ewald(emu_engine)


def test_geometry_loop_calls_check_their_state(emu_engine):
    """The geometry-loop entry points refuse a slot in the wrong state."""
    cell, f, rho_u, _ = cases.golden_case("wt_al4_displaced")
    s = cases.engine_slot(emu_engine, f, cell)  # tables set from the host: no ions known to the slot
    try:
        with pytest.raises(native.OfdftError) as ei:
            emu_engine.ewald(s, 4)
        assert ei.value.code == 1
        with pytest.raises(native.OfdftError) as ei:
            emu_engine.start_solve(s, None)  # no resident input yet
        assert ei.value.code == 1
        emu_engine.start_solve(s, rho_u)
        for call in (lambda: emu_engine.hold_density(s), lambda: emu_engine.ewald(s, 4),
                     lambda: emu_engine.set_input(s, rho_u)):
            with pytest.raises(native.OfdftError) as ei:
                call()
            assert ei.value.code == 4  # OFDFT_EBUSY while the solve runs
        emu_engine.cancel(s)
        emu_engine.hold_density(s)  # idle again: accepted
    finally:
        emu_engine.slot_destroy(s)


@pytest.mark.parametrize("n", [(1, 16, 16), (16, 16, 1024), (16, 13, 16)])
def test_grid_limits(emu_engine, n):
    cell, _, _, _ = cases.golden_case("wt_al4_displaced")
    with pytest.raises(native.OfdftError) as ei:
        emu_engine.slot_create(n, cell.lattice)
    assert ei.value.code == 1


def check_copy_tables(eng):
    """A slot whose tables are converted from another slot of the other
    precision (ofdft_slot_copy_tables) evaluates exactly like one given the
    same tables directly."""
    cell, f, _, _ = cases.golden_case("wgc_al4_fcc")
    s64 = cases.engine_slot(eng, f, cell, precision=native.FP64)
    s32 = cases.engine_slot(eng, f, cell, precision=native.FP32)
    c32 = eng.slot_create(f.n, cell.lattice, kinetic=f.kinetic, lam=f.lam, mu=f.mu, alpha=f.alpha, beta=f.beta,
                          rho_s=f.rho_s, precision=native.FP32)
    c64 = eng.slot_create(f.n, cell.lattice, kinetic=f.kinetic, lam=f.lam, mu=f.mu, alpha=f.alpha, beta=f.beta,
                          rho_s=f.rho_s, precision=native.FP64)
    try:
        eng.copy_tables(c32, s64)
        eng.copy_tables(c64, s64)
        rho = cases.random_density(f.n, cell.num_electrons, cell.vol, seed=21)
        for a, b in ((s32, c32), (s64, c64)):
            pa, ea = eng.calculate_potential_plus(a, rho)
            pb, eb = eng.calculate_potential_plus(b, rho)
            assert np.array_equal(pa, pb) and np.array_equal(ea, eb)
    finally:
        for s in (s64, s32, c32, c64):
            eng.slot_destroy(s)


def test_copy_tables(emu_engine):
    check_copy_tables(emu_engine)
