"""Density files (profess_b200.densityfile): the .den record layout, exact
round trips, ReadDensity's interpolation against the oracle's loops, and a
solve resumed from a written density (host-emulation build)."""
import re

import numpy as np
import pytest

import cases
from oracle import densityfile as odf
from profess_b200 import densityfile as df


def _rho(shape, seed=0):
    r = np.random.default_rng(seed).uniform(0.01, 0.05, size=shape)
    return np.asfortranarray(r)


def test_record_layout_and_round_trip(tmp_path):
    rho = _rho((5, 4, 3))
    rho[0, 0, 0] = 0.0
    p = str(tmp_path / "a.den")
    df.write_density(p, rho)
    raw = open(p, "rb").read()
    assert len(raw) == df.RECL * (4 + rho.size)
    recs = [raw[k * 27:(k + 1) * 27] for k in range(4 + rho.size)]
    assert recs[0] == b"x-dimension:             5\n" and recs[3] == b"# of spins:              1\n"
    assert all(re.fullmatch(rb"[ -]\.\d{20}E[+-]\d\d\n", r) for r in recs[4:])
    back = df.read_density_file(p)
    assert back.shape == (5, 4, 3, 1) and np.array_equal(back[..., 0], rho)


def test_e26_20_matches_fortran_form():
    assert df._e26_20(0.0123) == " .12300000000000000169E-01"  # the double's own decimal digits
    assert df._e26_20(0.375) == " .37500000000000000000E+00"
    assert df._e26_20(-1234.5) == "-.12345000000000000000E+04"
    assert float(df._e26_20(1.0 / 3.0)) == 1.0 / 3.0


def test_records_keep_their_length_at_the_exponent_limits(tmp_path):
    """A vacuum value below 1e-99 is written as zero (a three-digit exponent
    would lengthen the record); values that E26.20 cannot hold are refused."""
    assert df._e26_20(1e-120) == " .00000000000000000000E+00"
    assert df._e26_20(-3e-100) == " .00000000000000000000E+00"
    assert df._e26_20(1e-99).endswith("E-98") and float(df._e26_20(1e-99)) == 1e-99
    rho = _rho((3, 2, 2), seed=2)
    rho[1, 0, 0] = 1e-130
    p = str(tmp_path / "v.den")
    df.write_density(p, rho)
    assert len(open(p, "rb").read()) == df.RECL * (4 + rho.size)
    back = df.read_density_file(p)[..., 0]
    assert back[1, 0, 0] == 0.0 and np.array_equal(np.delete(back.ravel(order="F"), 1),
                                                    np.delete(rho.ravel(order="F"), 1))
    for bad in (np.nan, np.inf, -np.inf, 2e99):
        with pytest.raises(ValueError):
            df._e26_20(bad)
        rho[0, 1, 0] = bad
        with pytest.raises(ValueError):
            df.write_density(str(tmp_path / "bad.den"), rho)


@pytest.mark.parametrize("grid,repeat", [((5, 4, 3), (1, 1, 1)), ((10, 4, 6), (2, 1, 2)),
                                         ((8, 7, 6), (1, 1, 1)), ((9, 4, 5), (2, 1, 1))])
def test_read_matches_oracle(tmp_path, grid, repeat):
    f = _rho((5, 4, 3), seed=1)
    p = str(tmp_path / "b.den")
    df.write_density(p, f)
    got = df.read_density(p, grid, 12, 110.0, repeat)
    want = odf.read_density_loops(f, grid, 12, 110.0, repeat)
    assert np.abs(got - want).max() <= 1e-14 * np.abs(want).max()
    assert abs(got.sum() * 110.0 / got.size - 12) < 1e-12


def test_solve_resumes_from_a_written_density(emu_engine, tmp_path):
    cell, f, rho_u, _ = cases.golden_case("wt_al4_displaced")
    s = cases.engine_slot(emu_engine, f, cell)
    try:
        rho, e, st = emu_engine.proj_norm_rho_minimization(s, rho_u)
        p = str(tmp_path / "c.den")
        df.write_density(p, rho)
        rho2 = df.read_density(p, f.n, cell.num_electrons, cell.vol)
        assert np.abs(rho2 - rho).max() < 1e-12 * rho.max()
        _, e2, st2 = emu_engine.proj_norm_rho_minimization(s, rho2)
        # the energy criterion needs two iterations to see the change: 24 against 48 evaluations
        assert st2["num_evals"] <= st["num_evals"] // 2 and abs(e2[0] - e[0]) < 1e-7
    finally:
        emu_engine.slot_destroy(s)


def test_two_spin_file_is_refused(tmp_path):
    rho = _rho((3, 3, 2))
    p = str(tmp_path / "s.den")
    df.write_density(p, rho)
    raw = bytearray(open(p, "rb").read())
    raw[27 * 3:27 * 4] = b"# of spins:              2\n"
    open(p, "wb").write(bytes(raw) + bytes(raw[27 * 4:]))
    with pytest.raises(ValueError):
        df.read_density(p, (3, 3, 2), 12, 100.0)
