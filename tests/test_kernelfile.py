"""WT kernel files (profess_b200.kernelfile): round trip, the restart
interpolation against the oracle's bisection loops, and an evaluation with a
kernel read from a file against the kernel built from LindG."""
import numpy as np

import cases
from oracle import cellsetup as cs
from oracle import kedf_kernels as kk
from oracle import kernelfile as okf
from oracle.consts import PI
from profess_b200 import kernelfile as kf


def _table(nq=8001, eta_max=8.0):
    eta = np.linspace(0.0, eta_max, nq)
    return eta, kk.lind_g(eta, 1.0, 1.0)


def test_round_trip(tmp_path):
    eta, w = _table(101)
    p = str(tmp_path / "wt.ker")
    kf.write_wt_kernel_file(p, 0.9, 0.027, eta, w)
    t, k, r, e2, w2 = kf.read_wt_kernel_file(p)
    assert (t, k, r) == (kf.WT_TYPE, 0.9, 0.027)
    assert np.array_equal(e2, eta) and np.array_equal(w2, w)


def test_interpolation_matches_oracle_and_lindg(tmp_path):
    cell, f, _, _ = cases.golden_case("wt_al4_displaced")
    rho0 = cell.num_electrons / cell.vol
    kfermi = (3 * PI ** 2 * rho0) ** (1 / 3)
    coef = 5.0 / (9.0 * f.alpha * f.beta * rho0 ** (f.alpha + f.beta - 5.0 / 3.0))
    eta, w = _table()
    p = str(tmp_path / "wt.ker")
    kf.write_wt_kernel_file(p, kfermi, rho0, eta, w)
    qt = cs.q_table(cell.recip, *f.n)
    got = kf.wt_kernel_from_file(p, qt, kfermi, coef)
    assert np.array_equal(got, okf.wt_kernel_loops(eta, w, qt, kfermi, coef))
    exact = kk.wt_kernel(qt, rho0, f.alpha, f.beta, 1.0, 1.0)
    assert np.abs(got - exact).max() < 1e-4 * np.abs(exact).max()


def test_evaluation_with_a_kernel_file(emu_engine, tmp_path):
    cell, f, _, _ = cases.golden_case("wt_al4_displaced")
    rho0 = cell.num_electrons / cell.vol
    kfermi = (3 * PI ** 2 * rho0) ** (1 / 3)
    coef = 5.0 / (9.0 * f.alpha * f.beta * rho0 ** (f.alpha + f.beta - 5.0 / 3.0))
    eta, w = _table(20001)
    p = str(tmp_path / "wt.ker")
    kf.write_wt_kernel_file(p, kfermi, rho0, eta, w)
    s = cases.engine_slot(emu_engine, f, cell)
    try:
        rho = cases.random_density(f.n, cell.num_electrons, cell.vol, seed=2)
        _, e_built = emu_engine.calculate_potential_plus(s, rho)
        emu_engine.set_kernel(s, kf.wt_kernel_from_file(p, cs.q_table(cell.recip, *f.n), kfermi, coef)[None])
        _, e_file = emu_engine.calculate_potential_plus(s, rho)
        # linear interpolation on an eta spacing of 4e-4 (with LindG's log kink at eta = 1): 6e-8
        assert abs(e_file[8] - e_built[8]) < 1e-6 * abs(e_built[8])
    finally:
        emu_engine.slot_destroy(s)


def test_table_too_short_is_refused(tmp_path):
    import pytest
    eta, w = _table(101, eta_max=1.5)
    p = str(tmp_path / "short.ker")
    kf.write_wt_kernel_file(p, 1.0, 0.03, eta, w)
    with pytest.raises(ValueError):
        kf.wt_kernel_from_file(p, np.array([[[0.5, 4.0]]]), 1.0, 1.0)  # eta = 2 > 1.5
