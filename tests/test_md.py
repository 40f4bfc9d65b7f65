"""NVE molecular dynamics of replicas on the engine (profess_b200.md) against
the oracle's restatement of RunNVE (oracle/md.py), on the host-emulation
build (CPU); test_gpu_md.py repeats them on the CUDA build."""
import numpy as np

from oracle import cellsetup as cs
from oracle import functional as fn
from oracle import md as omd
from oracle import ntn
from profess_b200 import md, native, workloads as wl

DT = 40.0  # a.u. of time (~0.97 fs)


def _cells():
    c = wl.fcc_al((1, 1, 1), sigma_ang=0.05, grid=(20, 20, 20), seed=3)
    mx, vals = wl.heine_abarenkov_table(3.0, 1.15, 0.1)
    ocell = cs.Cell(lattice=c.lattice, frac=c.frac, species_of_ion=c.species_of_ion,
                    species=[cs.species_from_table(mx, vals, "Al")])
    return c, ocell


def _wrap(d):
    return d - np.rint(d)


def check_nve_matches_oracle(eng, nsteps=3):
    c, ocell = _cells()
    v0 = md.initial_velocities(c, 600.0, seed=4)
    opts = native.ntn_options(conv_check=native.CONV_POT, pot_tol=1.0e-6)
    run = md.NVE(eng, [c], DT, velocities=[v0], opts=opts)
    try:
        run.run(nsteps)
        rep = run.reps[0]
        ref = omd.run_nve(ocell, c.grid, v0, DT, nsteps, ntn.NtnOptions(conv_check="POT", pot_tol=1.0e-6))
        last = ref[-1]
        assert np.abs(_wrap(rep.cell.frac - last.frac)).max() < 1e-10
        assert np.abs(rep.vel - last.vel).max() < 1e-10 * np.abs(last.vel).max() + 1e-14
        assert abs(float(rep.energy[0]) - last.energy) < 1e-8
        assert np.abs(rep.forces - last.forces).max() < 1e-8
        cons = [h["conserved"] for h in rep.history]
        assert max(cons) - min(cons) < 1e-4  # Ha, 3 steps of ~1 fs
        assert all(abs(h["conserved"] - s.conserved) < 1e-8 for h, s in zip(rep.history, ref[1:]))
    finally:
        run.close()


def test_atomic_masses():
    assert abs(md.atomic_mass("Al") - 49184.3) < 1.0  # 26.98 amu in electron masses
    assert md.atomic_mass("Al") == omd.atomic_mass("Al")


def test_initial_velocities_temperature_and_momentum():
    c, _ = _cells()
    v = md.initial_velocities(c, 600.0, seed=1)
    m = md.masses_of(c)
    assert np.abs((m[:, None] * v).sum(axis=0)).max() < 1e-12
    ke = 0.5 * float((m[:, None] * v * v).sum())
    assert abs(ke - 1.5 * c.nion * 600.0 * md.BOLTZMANN) < 1e-12


def test_nve_matches_oracle(emu_engine):
    check_nve_matches_oracle(emu_engine)


def test_nve_replicas_batched_as_alone(emu_engine):
    """Two replicas stepped together give the same trajectories as each alone."""
    cells = [wl.fcc_al((1, 1, 1), sigma_ang=0.05, grid=(16, 16, 16), seed=s) for s in (1, 2)]
    vs = [md.initial_velocities(c, 300.0, seed=s) for s, c in enumerate(cells)]
    alone = []
    for c, v in zip(cells, vs):
        r = md.NVE(emu_engine, [c], DT, velocities=[v])
        r.run(2)
        alone.append((r.reps[0].cell.frac.copy(), r.reps[0].vel.copy(), float(r.reps[0].energy[0])))
        r.close()
    both = md.NVE(emu_engine, cells, DT, velocities=vs)
    try:
        both.run(2)
        for rep, (fr, v, e) in zip(both.reps, alone):
            assert np.array_equal(rep.cell.frac, fr) and np.array_equal(rep.vel, v) and float(rep.energy[0]) == e
    finally:
        both.close()


def test_nvt_matches_oracle(emu_engine):
    check_nvt_matches_oracle(emu_engine)


def check_nvt_matches_oracle(eng):
    """Nose-Hoover NVT (RunNVT) on the engine against the oracle's restatement."""
    c, ocell = _cells()
    v0 = md.initial_velocities(c, 300.0, seed=7)
    opts = native.ntn_options(conv_check=native.CONV_POT, pot_tol=1.0e-6)
    q = 2000.0
    run = md.NVT(eng, [c], DT, q_mass=q, temperature_k=900.0, velocities=[v0], opts=opts)
    try:
        run.run(3)
        rep = run.reps[0]
        ref = omd.run_nvt(ocell, c.grid, v0, DT, 3, ntn.NtnOptions(conv_check="POT", pot_tol=1.0e-6), q,
                          900.0 * md.BOLTZMANN)
        fr, vel, energy, h = ref[-1]
        assert np.abs(_wrap(rep.cell.frac - fr)).max() < 1e-10
        assert np.abs(rep.vel - vel).max() < 1e-10 * np.abs(vel).max()
        assert abs(float(rep.energy[0]) - energy) < 1e-8
        assert all(abs(hh["conserved"] - r[3]) < 1e-8 for hh, r in zip(rep.history, ref))
        # the thermostat heats the 300 K start towards 900 K
        assert rep.history[-1]["temperature"] > 300.0
    finally:
        run.close()


def test_yoshida_weights_sum_to_one():
    for n in (1, 3, 5):
        assert abs(md.yoshida_coefficients(n).sum() - 1.0) < 1e-15


NPT_Q, NPT_B, NPT_P = 2.0e3, 2.0e5, 1.0e-5


def check_npt_matches_oracle(eng, nsteps=3, wgc=False):
    """Full-cell NPT (NPTFullCell) on the engine, with the device stress and
    the device lattice refresh, against the oracle's restatement: the same
    lattice, positions, energy and conserved quantity after every step.  With
    wgc, the cell runs the second-order WGC functional (its kernel rebuilt
    on the device after every lattice move, WGCStress)."""
    c, ocell = _cells()
    extra = {}
    if wgc:
        c.kinetic, c.alpha, c.beta = native.KEDF_WGC, (5 + 5 ** 0.5) / 6, (5 - 5 ** 0.5) / 6
        extra = dict(alpha=c.alpha, beta=c.beta, kinetic=fn.KEDF_WGC, gamma=c.gamma)
    v0 = md.initial_velocities(c, 600.0, seed=4)
    opts = native.ntn_options(conv_check=native.CONV_POT, pot_tol=1.0e-6)
    run = md.NPT(eng, [c], DT, NPT_Q, NPT_B, 600.0, NPT_P, velocities=[v0], opts=opts)
    try:
        run.run(nsteps)
        rep = run.reps[0]
        ref = omd.run_npt(ocell, c.grid, v0, DT, nsteps, ntn.NtnOptions(conv_check="POT", pot_tol=1.0e-6),
                          NPT_Q, NPT_B, 600.0 * md.BOLTZMANN, NPT_P, **extra)
        lat, frac, energy, cons, vol = ref[-1]
        assert np.abs(rep.cell.lattice - lat).max() < 1e-11
        assert np.abs(_wrap(rep.cell.frac - frac)).max() < 1e-10
        assert abs(float(rep.energy[0]) - energy) < 1e-8
        for h, r in zip(rep.history, ref[1:]):
            assert abs(h["conserved"] - r[3]) < 1e-8 and abs(h["volume"] - r[4]) < 1e-9
        assert abs(ref[-1][4] - ref[0][4]) > 1e-3  # the cell did move
    finally:
        run.close()


def test_npt_matches_oracle(emu_engine):
    check_npt_matches_oracle(emu_engine)


def test_npt_wgc_matches_oracle(emu_engine):
    check_npt_matches_oracle(emu_engine, nsteps=2, wgc=True)


def test_box_constraint():
    m = np.arange(9.0).reshape(3, 3) + 1.0
    assert np.array_equal(md.box_constraint(m, -1), m)
    assert np.array_equal(md.box_constraint(m, 1), np.diag(np.diag(m)))
    assert np.array_equal(md.box_constraint(m, 4), np.diag([1.0, 0.0, 9.0]))
