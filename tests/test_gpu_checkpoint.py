"""Checkpoint and resume of device-resident densities in the reference's .den
format (GPU): a solve stopped part-way, its resident density written with
PrintDensity's layout (Source/Output.f90:876-953) and read back with
ReadDensity's (Source/ReadIonFile.f90:1054-1314), resumes to the same result
as a resume from the density still on the device.  The E26.20 records hold a
double exactly, so the two resumed solves are bitwise equal; both converge to
the energy of an uninterrupted solve within 1e-10 Ha."""
import numpy as np
import pytest

from profess_b200 import cell as pcell
from profess_b200 import densityfile as df
from profess_b200 import native, workloads as wl



def check_checkpoint(eng, tmp_path, c, prec):
    s = pcell.setup_slot(eng, c, prec)
    opts = native.ntn_options(conv_check=native.CONV_POT, pot_tol=1e-7 if prec == native.FP64 else 3e-5,
                              max_iter=300, stall_line=6)
    try:
        rho0 = wl.initial_density(c, seed=3)
        _, e_full, _ = eng.proj_norm_rho_minimization(s, rho0, opts)
        # stop a solve part-way: the density stays on the device
        eng.start_solve(s, rho0, opts)
        eng.run(24)
        eng.cancel(s)
        mid = eng.download(s, 0) ** 2  # phi^2, the resident density
        path = str(tmp_path / "mid.den")
        df.write_density(path, mid)
        back = df.read_density(path, c.grid, c.num_electrons, c.vol)
        # the checkpoint holds the resident density to the last bit; reading
        # renormalises it to the cell's electron count (a factor 1 + O(1e-15)
        # for an FP64 slot, 1 + O(1e-8) for an FP32 one)
        raw = df.read_density_file(path)[..., 0]
        assert np.array_equal(raw, mid)
        scale = c.num_electrons / (mid.sum() * c.vol / mid.size)
        assert np.abs(back - mid * scale).max() <= 1e-14 * np.abs(mid).max()
        assert abs(scale - 1.0) < (1e-12 if prec == native.FP64 else 1e-6)
        eng.hold_density(s)
        eng.start_solve(s, None, opts)
        while eng.run(8):
            pass
        r_dev, e_dev, st_dev = eng.result(s)
        _, e_file, st_file = eng.proj_norm_rho_minimization(s, raw, opts)
        assert st_dev["outcome"] in (0, 2) and st_file["outcome"] in (0, 2)
        assert np.array_equal(e_dev, e_file) and st_dev["num_evals"] == st_file["num_evals"]
        if prec == native.FP64:
            assert abs(e_dev[0] - e_full[0]) < 1e-10
    finally:
        eng.slot_destroy(s)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [native.FP64, native.FP32])
def test_checkpoint_and_resume(gpu_engine, tmp_path, prec):
    check_checkpoint(gpu_engine, tmp_path, wl.fcc_al((2, 2, 2), sigma_ang=0.05, grid=(48, 48, 48), seed=7), prec)


def test_checkpoint_and_resume_emulated(emu_engine, tmp_path):
    """The same on the host emulation of the kernels (CPU), on a 16^3 cell."""
    check_checkpoint(emu_engine, tmp_path, wl.fcc_al((1, 1, 1), sigma_ang=0.05, grid=(16, 16, 16), seed=7),
                     native.FP64)
