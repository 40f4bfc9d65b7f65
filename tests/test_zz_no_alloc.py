"""The allocation-free evaluation entry point against the engine's own.

ofdft_calculate_potential_plus_noalloc serves callers that cannot allocate
device memory (a host code inside a device-memory pool it does not own, or
under a memory budget fixed before the solve): its scratch is a static array
inside the library.  This test gives it device buffers that the test itself
allocates and checks two calls in a row (two different densities) against
ofdft_calculate_potential_plus at the tolerances of the other GPU parity
tests (potential 1e-11 relative, energy terms 1e-10 Ha), and the second call
against the oracle as well.  The grids reach the documented limits: 64^3
(262144 points), a 128-point axis (128 x 128 x 16), and alpha != beta (four
spectra in the scratch instead of three)."""
import ctypes

import numpy as np
import pytest

import cases
from oracle import functional as ofn
from profess_b200 import native

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("n,alpha,beta", [(None, 5 / 6, 5 / 6), ((32, 30, 27), 5 / 6, 5 / 6),
                                          ((64, 64, 64), 5 / 6, 5 / 6), ((128, 128, 16), 5 / 6, 5 / 6),
                                          ((40, 36, 30), 1.2, 0.45)])
def test_noalloc_matches_engine(n, alpha, beta):
    import torch
    torch.cuda.set_device(0)
    cell, f, _, _ = cases.golden_case("wt_al4_displaced")
    if n is not None or alpha != beta:
        f = cases.functional_for(cell, n or f.n, 4, alpha, beta)
    lib = native.load_library()
    fn = lib.ofdft_calculate_potential_plus_noalloc
    fn.argtypes = [ctypes.POINTER(native.CellDesc), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    eng = native.Engine(lib)
    try:
        slot = cases.engine_slot(eng, f, cell)
        desc = native.CellDesc(f.n[0], f.n[1], f.n[2],
                               (ctypes.c_double * 9)(*np.asarray(cell.lattice).ravel(order="F")),
                               4, f.lam, f.mu, f.alpha, f.beta, 2.7, 0.0, f.rho_s, f.ion_ion, native.FP64)
        d_kern = _dev(f.kernel[0])
        d_vion = _dev(f.ion_pot)
        d_pot = torch.zeros(int(np.prod(f.n)), dtype=torch.float64, device="cuda")
        for call, seed in enumerate((11, 12)):
            rho = cases.random_density(f.n, cell.num_electrons, cell.vol, seed=seed)
            d_rho = _dev(rho)
            et = np.zeros(9)
            torch.cuda.synchronize()
            rc = fn(ctypes.byref(desc), d_rho.data_ptr(), d_kern.data_ptr(), d_vion.data_ptr(), 1,
                    d_pot.data_ptr(), et.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None)
            assert rc == 0, lib.ofdft_last_error().decode()
            pot = d_pot.cpu().numpy().reshape(f.n, order="F")
            pot_e, et_e = eng.calculate_potential_plus(slot, rho)
            assert np.abs(pot - pot_e).max() / np.abs(pot_e).max() < 1e-11, "call %d" % call
            assert np.abs(et - et_e).max() < 1e-10, "call %d" % call
            if call == 1:
                pot_o, et_o = ofn.calculate_potential_plus(f, rho)
                assert np.abs(pot - pot_o).max() / np.abs(pot_o).max() < 1e-11
                assert np.abs(et - et_o).max() < 1e-10
    finally:
        eng.close()


def test_noalloc_rejects_oversize():
    lib = native.load_library()
    fn = lib.ofdft_calculate_potential_plus_noalloc
    fn.argtypes = [ctypes.POINTER(native.CellDesc), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    lat = (ctypes.c_double * 9)(20, 0, 0, 0, 20, 0, 0, 0, 20)
    desc = native.CellDesc(96, 96, 96, lat, 4, 1.0, 1.0, 5 / 6, 5 / 6, 2.7, 0.0, 0.0, 0.0, native.FP64)
    rc = fn(ctypes.byref(desc), 1, 1, 1, 1, 1, None, None)  # rejected before any pointer is used
    assert rc == 1 and b"too large" in lib.ofdft_last_error()
