"""Host-side set-up logic against the oracle (CPU): grid sizing, recpot
reading, the Heine-Abarenkov workload tables, Ewald, the WGC kernel ODE, footprints."""
import numpy as np
import pytest

import cases
from oracle import cellsetup as cs
from oracle import ewald as oew
from oracle import kedf_kernels as kk
from oracle.consts import HARTREE_TO_EV
from profess_b200 import native, recpot, workloads as wl


@pytest.fixture(scope="module")
def lib():
    from profess_b200 import build
    return native.load_library(build.build_emu())


def test_constants_match_oracle():
    assert recpot.HARTREE_TO_EV == HARTREE_TO_EV


@pytest.mark.parametrize("ecut", [600.0, 900.0, 1500.0])
@pytest.mark.parametrize("name", ["wt_al4_displaced", "wgc_al4_fcc"])
def test_grid_size(lib, ecut, name):
    cell, _, _, _ = cases.golden_case(name)
    assert native.grid_size(lib, ecut / HARTREE_TO_EV, cell.lattice) == cs.size_system(ecut / HARTREE_TO_EV,
                                                                                        cell.lattice)


def test_recpot_reader_matches_oracle():
    z = np.load(cases.GOLDEN + "/al_hc_recpot.npz")
    a = recpot.species_from_table(float(z["max_g"]), z["values"], "Al")
    b = cases.al_species()
    assert a.charge == b.charge == 3
    assert np.array_equal(a.pot_values, b.pot_values) and np.array_equal(a.vqs, b.vqs)
    assert np.abs(a.pot_dd - b.pot_dd).max() < 1e-9 * np.abs(b.pot_dd).max()


def test_recpot_text_round_trip():
    mx, vals = wl.heine_abarenkov_table(2.0, 1.3, 0.1)
    text = recpot.format_recpot(mx, vals, "HA Mg")
    sp = recpot.parse_recpot(text, "Mg")
    ref = recpot.species_from_table(mx, vals, "Mg")
    assert sp.charge == 2 and np.allclose(sp.pot_values, ref.pot_values, rtol=1e-15, atol=0)
    osp = cs.parse_recpot_text(text, "Mg")
    assert osp.charge == 2 and np.allclose(osp.vqs, sp.vqs, rtol=1e-15, atol=0)


def test_heine_abarenkov_tables_have_the_coulomb_tail():
    for z, rc in [(3, 1.15), (2, 1.3)]:
        mx, vals = wl.heine_abarenkov_table(float(z), rc, 0.1)
        sp = recpot.species_from_table(mx, vals)
        assert sp.charge == z
        # v(q) q^2 -> -4 pi Z as q -> 0 (the tail ReadPseudo infers Z from)
        q = np.arange(1, 6) * sp.max_g / (len(sp.pot_values) - 1)
        tail = sp.pot_values[1:6] * q ** 2
        assert np.all(np.abs(tail / (-4 * np.pi * z) - 1.0) < 1e-4)


def test_heine_abarenkov_table_is_the_transform_of_the_model_potential():
    """v(q) + 4 pi Z / q^2 = 4 pi int_0^rc r^2 (-A + Z/r) j0(qr) dr (quadrature)."""
    from profess_b200.recpot import BOHR, HARTREE_TO_EV
    z, rc, a = 2.0, 1.3, 0.1
    mx, vals = wl.heine_abarenkov_table(z, rc, a)
    v = vals / (BOHR ** 3 * HARTREE_TO_EV)
    x, w = np.polynomial.legendre.leggauss(64)
    r, wr = 0.5 * rc * (x + 1.0), 0.5 * rc * w
    for k in [0, 1, 7, 150, 2000, 15002]:
        q = 0.002 * k
        j0 = np.sinc(q * r / np.pi)
        short = 4 * np.pi * float(np.sum(wr * r * r * (-a + z / r) * j0))
        coul = 0.0 if k == 0 else -4 * np.pi * z / q ** 2
        assert abs(v[k] - coul - short) < 1e-10 * max(1.0, abs(coul))


@pytest.mark.parametrize("name", ["wt_al4_displaced", "wgc_al4_fcc"])
def test_ewald_matches_oracle(lib, name):
    cell, _, _, _ = cases.golden_case(name)
    e, f = native.ewald(lib, cell.lattice, cell.frac, cell.charges(), True)
    eo, fo = oew.ewald(cell.lattice, cell.frac, cell.charges(), True)
    assert abs(e - eo) < 1e-11 and np.abs(f - fo).max() < 1e-11


def test_ewald_supercell_extensive(lib):
    c1 = wl.fcc_al((1, 1, 1))
    c2 = wl.fcc_al((2, 2, 2))
    e1, _ = native.ewald(lib, c1.lattice, c1.frac, c1.charges())
    e2, _ = native.ewald(lib, c2.lattice, c2.frac, c2.charges())
    assert abs(e2 - 8 * e1) < 1e-9 * abs(e2)


def test_wgc_ode_tables(lib):
    a, b = 1.2060113295832983, 0.46065533708336838
    t = native.wgc_radial_tables(lib, a, b, 2.7)
    r = kk.wgc_radial_tables(a, b, 2.7)
    assert np.array_equal(t[0], r[0])
    for x, y in zip(t[1:], r[1:]):
        assert np.abs(x - y).max() <= 1e-5 * (1 + np.abs(y).max())


def test_workload_configs():
    c1 = wl.config_cell(1)
    assert c1.nion == 4 and c1.grid == (32, 32, 32) and c1.num_electrons == 12
    c2 = wl.config_cell(2)
    assert c2.nion == 256 and c2.grid == (96, 96, 96)
    for i in range(6):
        c3 = wl.config_cell(3, index=i)
        n = round((c3.nion / 4) ** (1 / 3))
        assert c3.nion in (32, 108, 256, 500) and c3.grid == (24 * n,) * 3
    c4 = wl.config_cell(4)
    assert c4.nion == 1152 and c4.grid == (160, 160, 256) and c4.kinetic == 5
    assert abs(c4.alpha + c4.beta - 5.0 / 3.0) < 1e-15
    rho = wl.initial_density(c2)
    assert abs(rho.sum() * c2.vol / rho.size - c2.num_electrons) < 1e-9


def test_footprint_grows_with_grid(lib):
    small = native.slot_footprint(lib, (32, 32, 32), 4, 5 / 6, 5 / 6, native.FP64)
    big = native.slot_footprint(lib, (96, 96, 96), 4, 5 / 6, 5 / 6, native.FP64)
    f32 = native.slot_footprint(lib, (96, 96, 96), 4, 5 / 6, 5 / 6, native.FP32)
    wgc = native.slot_footprint(lib, (96, 96, 96), 5, 1.2, 0.46, native.FP64)
    assert small < big and f32 < big < wgc
    assert big > 96 ** 3 * 8 * 10
