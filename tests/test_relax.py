"""QuickMin relaxation of cells on the engine (profess_b200.relax) against the
oracle's restatement of QuickMinOptimization (oracle/relax.py), on the
host-emulation build (CPU); test_gpu_relax.py repeats it on the CUDA build."""
import numpy as np
import pytest

from oracle import cellsetup as cs
from oracle import ntn
from oracle import relax as orelax
from profess_b200 import native, relax, workloads as wl


def _cell(seed=3, grid=(16, 16, 16)):
    c = wl.fcc_al((1, 1, 1), sigma_ang=0.1, grid=grid, seed=seed)
    mx, vals = wl.heine_abarenkov_table(3.0, 1.15, 0.1)
    ocell = cs.Cell(lattice=c.lattice, frac=c.frac, species_of_ion=c.species_of_ion,
                    species=[cs.species_from_table(mx, vals, "Al")])
    return c, ocell


def check_quickmin_matches_oracle(eng, max_steps=12):
    c, ocell = _cell()
    opts = native.ntn_options(conv_check=native.CONV_POT, pot_tol=1.0e-6)
    qm = relax.QuickMin(eng, [c], max_steps=max_steps, opts=opts)
    try:
        st = qm.run()[0]
        frac, energy, forces, hist = orelax.quickmin(ocell, c.grid, ntn.NtnOptions(conv_check="POT", pot_tol=1.0e-6),
                                                     max_steps=max_steps)
        assert [h["undone"] for h in st.history] == [h[4] for h in hist]
        assert [h["time_step"] for h in st.history] == [h[3] for h in hist]
        d = st.cell.frac - frac
        assert np.abs(d - np.rint(d)).max() < 1e-9
        assert abs(float(st.energy[0]) - energy) < 1e-8
        assert np.abs(st.forces - forces).max() < 1e-8
        # the run takes kept and undone moves, and lowers the largest force
        assert any(h["undone"] for h in st.history) and not all(h["undone"] for h in st.history)
        assert st.best_force < 0.5 * st.initial_max_force
    finally:
        qm.close()


def test_quickmin_matches_oracle(emu_engine):
    check_quickmin_matches_oracle(emu_engine)


def test_quickmin_batch_same_as_alone(emu_engine):
    cells = [_cell(seed=s, grid=(12, 12, 12))[0] for s in (1, 2)]
    alone = []
    for c in cells:
        q = relax.QuickMin(emu_engine, [c], max_steps=6)
        st = q.run()[0]
        alone.append((st.cell.frac.copy(), float(st.energy[0]), [h["time_step"] for h in st.history]))
        q.close()
    q = relax.QuickMin(emu_engine, cells, max_steps=6)
    try:
        for st, (fr, e, ts) in zip(q.run(), alone):
            assert np.array_equal(st.cell.frac, fr) and float(st.energy[0]) == e
            assert [h["time_step"] for h in st.history] == ts
    finally:
        q.close()


# ------------------------------------------------------------------ CG2
# TOTAL ENERGY lines of the reference's CG2 relaxation of this cell
# (test/optIon/sampleoutput/displaced.out:123-938), eV: every density solve.
REF_CG2_TRACE_EV = [-231.1425327622, -231.2770513588, -231.6147260670, -231.6471183146, -231.6860136007,
                    -231.6996685913, -231.7083720964, -231.7111562797, -231.7116104934, -231.7118205898,
                    -231.7118261145, -231.7118465883, -231.7118498940]


def test_oracle_cg2_reproduces_the_reference_trace():
    """The oracle's CG2 takes the reference's 13 density solves; their energies
    agree to 1e-4 eV (each solve converges to dE < 1e-6 Ha)."""
    import cases
    from oracle import cg2 as ocg2
    from oracle.consts import HARTREE_TO_EV
    cell, f, _, _ = cases.golden_case("wt_al4_displaced")
    _, trace, _ = ocg2.cg2(cell, f.n, ntn.NtnOptions())
    assert len(trace) == len(REF_CG2_TRACE_EV)
    assert np.abs(np.array(trace) * HARTREE_TO_EV - REF_CG2_TRACE_EV).max() < 1e-4


def check_cg2_matches_oracle(eng):
    import cases
    from oracle import cg2 as ocg2
    cell, f, _, _ = cases.golden_case("wt_al4_displaced")
    from profess_b200 import recpot
    z = np.load(cases.GOLDEN + "/al_hc_recpot.npz")
    sp = recpot.species_from_table(float(z["max_g"]), z["values"], "Al")
    c = wl.Cell(name="displaced", lattice=cell.lattice, frac=cell.frac, species_of_ion=cell.species_of_ion,
                species=[sp], grid=tuple(f.n))
    run = relax.CG2(eng, [c])
    try:
        run.run()
        frac, trace, forces = ocg2.cg2(cell, f.n, ntn.NtnOptions())
        assert len(run.traces[0]) == len(trace)
        assert np.abs(np.array(run.traces[0]) - trace).max() < 1e-9
        d = run.states[0].cell.frac - frac
        # the last steps are ~10 bohr per Ha/bohr of force along forces of ~1e-4, so the
        # positions carry the solves' convergence noise: 3e-8 (fractional) on the emulator
        assert np.abs(d - np.rint(d)).max() < 2e-7
    finally:
        run.close()


def test_cg2_matches_oracle(emu_engine):
    check_cg2_matches_oracle(emu_engine)


def _rosenbrock(x):
    f = float(((1.0 - x[:-1]) ** 2 + 100.0 * (x[1:] - x[:-1] ** 2) ** 2).sum())
    g = np.zeros_like(x)
    g[:-1] = -2.0 * (1.0 - x[:-1]) - 400.0 * x[:-1] * (x[1:] - x[:-1] ** 2)
    g[1:] += 200.0 * (x[1:] - x[:-1] ** 2)
    return f, g


def test_lbfgs_matches_oracle_on_rosenbrock():
    """The engine's LBFGS (reverse communication) and the oracle's work-array
    restatement take the same iterates, line-search trials included, on a
    function whose searches bracket, interpolate and restart."""
    from oracle import lbfgs as olb
    for n, seed in ((2, 0), (6, 1), (12, 2)):
        x0 = np.random.default_rng(seed).uniform(-1.5, 1.5, n)
        xa, xb = x0.copy(), x0.copy()
        la, lb = relax.Lbfgs(), olb.LbfgsRC(n)
        fa, ga = _rosenbrock(xa)
        ia = ib = 0
        calls = 0
        while True:
            xa, ia = la.call(xa, fa, ga, ia)
            ib = lb.call(xb, fa, ga, ib)
            assert ia == ib
            np.testing.assert_array_equal(xa, xb)
            fa, ga = _rosenbrock(xa)
            calls += 1
            if ia <= 0 or calls > 400:
                break
        assert ia == 0 and np.abs(xa - 1.0).max() < 1e-3, (n, ia, xa)


@pytest.mark.filterwarnings("ignore:invalid value")
def test_mcstep_matches_oracle():
    """MCSTEP on random states, inconsistent ones included (NaN steps where a
    cubic has no real minimiser, as under IEEE arithmetic)."""
    from oracle import lbfgs as olb
    rng = np.random.default_rng(5)
    same = lambda a, b: a == b or (a != a and b != b)  # noqa: E731
    for _ in range(2000):
        stx, sty = 0.0, float(rng.uniform(0.1, 2.0))
        args = (stx, float(rng.normal()), -abs(float(rng.normal())) - 1e-3, sty, float(rng.normal()),
                float(rng.normal()), float(rng.uniform(0.05, 3.0)), float(rng.normal()), float(rng.normal()),
                bool(rng.integers(2)), 0.0, 4.0)
        ra, rb = relax.mt_step(*args), olb.mcstep(*args)
        assert all(same(a, b) for a, b in zip(ra, rb)), (args, ra, rb)


def check_bfgs_matches_oracle(eng):
    """IonLBFGS on the engine against the oracle, from the displaced Al4 cell:
    the same energy after every density solve, the same final geometry."""
    import cases
    from oracle import lbfgs as olb
    cell, f, _, _ = cases.golden_case("wt_al4_displaced")
    from profess_b200 import recpot
    z = np.load(cases.GOLDEN + "/al_hc_recpot.npz")
    sp = recpot.species_from_table(float(z["max_g"]), z["values"], "Al")
    c = wl.Cell(name="displaced", lattice=cell.lattice, frac=cell.frac, species_of_ion=cell.species_of_ion,
                species=[sp], grid=tuple(f.n))
    run = relax.BFGS(eng, [c])
    try:
        run.run()
        frac, trace, forces = olb.bfgs(cell, f.n, ntn.NtnOptions())
        assert len(run.traces[0]) == len(trace)
        assert np.abs(np.array(run.traces[0]) - trace).max() < 1e-9
        assert trace[-1] < trace[0] - 1e-2
        assert relax._max_force(run.states[0].forces) < relax.FORCE_CUTOFF
        assert np.abs(run.states[0].cell.frac - frac).max() < 2e-7
    finally:
        run.close()


def test_bfgs_matches_oracle(emu_engine):
    check_bfgs_matches_oracle(emu_engine)


def check_bfgs_wgc_matches_oracle(eng):
    """IonLBFGS of a second-order WGC Al4 cell with displaced ions (the WGC
    kernel stays, the ion potential and Ewald sum follow the ions) against
    the oracle with the same functional."""
    import cases
    from oracle import functional as fn
    from oracle import lbfgs as olb
    from profess_b200 import recpot
    import dataclasses
    cell0, f, _, c = cases.golden_case("wgc_al4_fcc")
    shift = np.array([[0.012, -0.008, 0.005], [-0.006, 0.01, 0.0], [0.0, -0.004, -0.009], [0.007, 0.0, 0.006]])
    cell = dataclasses.replace(cell0, frac=np.mod(cell0.frac + shift, 1.0))
    z = np.load(cases.GOLDEN + "/al_hc_recpot.npz")
    sp = recpot.species_from_table(float(z["max_g"]), z["values"], "Al")
    wc = wl.Cell(name="al4_wgc", lattice=cell.lattice, frac=cell.frac, species_of_ion=cell.species_of_ion,
                 species=[sp], grid=tuple(f.n), kinetic=native.KEDF_WGC, alpha=c["alpha"], beta=c["beta"],
                 gamma=c["gamma"])
    run = relax.BFGS(eng, [wc])
    try:
        run.run()
        frac, trace, _ = olb.bfgs(cell, f.n, ntn.NtnOptions(), alpha_=c["alpha"], beta_=c["beta"],
                                  kinetic=fn.KEDF_WGC, gamma=c["gamma"])
        assert len(run.traces[0]) == len(trace) > 2
        assert np.abs(np.array(run.traces[0]) - trace).max() < 1e-9
        assert trace[-1] < trace[0] - 1e-4
        assert relax._max_force(run.states[0].forces) < relax.FORCE_CUTOFF
        assert np.abs(run.states[0].cell.frac - frac).max() < 2e-7
    finally:
        run.close()


def test_bfgs_wgc_matches_oracle(emu_engine):
    check_bfgs_wgc_matches_oracle(emu_engine)


def test_library_line_search_matches_oracle(emu_engine):
    """ofdft_dcsrch (the solver's Dcsrch) takes the same trial steps and ends
    with the same task as the oracle's Dcsrch on 1D functions."""
    from oracle.linesearch import Dcsrch
    codes = {"FG": native.LS_FG, "CONV": native.LS_CONV, "WARN": native.LS_WARN, "ERRO": native.LS_ERROR}
    funcs = [lambda a: ((a - 0.7) ** 2 - 0.3 * a, 2 * (a - 0.7) - 0.3),
             lambda a: (np.cos(3 * a) + 0.1 * a * a, -3 * np.sin(3 * a) + 0.2 * a),
             lambda a: (-np.exp(-a) * a, np.exp(-a) * (a - 1.0))]
    for fun in funcs:
        for stp0 in (0.05, 1.0, 5.0):
            for tols in ((1e-4, 0.9, 1e-10), (0.01, 0.1, 1e-10)):
                a = native.Dcsrch(emu_engine.lib, *tols, 1e-100, 1000.0)
                b = Dcsrch(*tols, 1e-100, 1000.0)
                sa = sb = stp0
                f, g = fun(0.0)
                ta, tb = native.LS_START, "START"
                for _ in range(40):
                    sa, ta = a.step(sa, f, g, ta)
                    sb, tb = b.step(sb, f, g, tb)
                    assert ta == codes[tb[:4]] and sa == sb, (ta, tb, sa, sb)
                    if ta != native.LS_FG:
                        break
                    f, g = fun(sa)


def check_gradient_cg_matches_oracle(eng):
    """GradientOptimization on the engine against the oracle from the
    displaced Al4 cell: the same energy after every density solve."""
    import cases
    from oracle import ioncg
    cell, f, _, _ = cases.golden_case("wt_al4_displaced")
    from profess_b200 import recpot
    z = np.load(cases.GOLDEN + "/al_hc_recpot.npz")
    sp = recpot.species_from_table(float(z["max_g"]), z["values"], "Al")
    c = wl.Cell(name="displaced", lattice=cell.lattice, frac=cell.frac, species_of_ion=cell.species_of_ion,
                species=[sp], grid=tuple(f.n))
    run = relax.GradientCG(eng, [c], max_steps=12)
    try:
        run.run()
        frac, trace, forces = ioncg.gradient_optimization(cell, f.n, ntn.NtnOptions(), max_steps=12)
        assert len(run.traces[0]) == len(trace)
        assert np.abs(np.array(run.traces[0]) - trace).max() < 1e-9
        assert trace[-1] < trace[0] - 1e-2
        d = run.states[0].cell.frac - frac
        assert np.abs(d - np.rint(d)).max() < 2e-7
    finally:
        run.close()


def test_gradient_cg_matches_oracle(emu_engine):
    check_gradient_cg_matches_oracle(emu_engine)
