"""The autotuner (ofdft_engine_tune) and pinned launch shapes
(ofdft_slot_set_shape): every shape it may pick computes the same potential
and energies as the oracle, a tuned shape is cached for the kind of cell and
given to later slots, and shapes out of range are refused.  On the host
emulation (CPU); test_gpu_features.py tunes on the GPU."""
import numpy as np
import pytest

import cases
from oracle import functional as fn
from profess_b200 import native

SHAPES = [dict(x_radix_cap=0, xfwd_row_pairs=1, xinv_row_pairs=1, yz_threads=0),
          dict(x_radix_cap=8, xfwd_row_pairs=3, xinv_row_pairs=2, yz_threads=512),
          dict(x_radix_cap=12, xfwd_row_pairs=5, xinv_row_pairs=7, yz_threads=256),
          dict(x_radix_cap=8, xfwd_row_pairs=16, xinv_row_pairs=9, yz_threads=0)]


def check_shapes_same_results(eng, name="wt_al4_displaced", prec=native.FP64, tol_pot=1e-11, tol_e=1e-10):
    cell, f, _, _ = cases.golden_case(name)
    s = cases.engine_slot(eng, f, cell, precision=prec)
    try:
        rho = cases.random_density(f.n, cell.num_electrons, cell.vol, seed=2)
        pot_o, et_o = fn.calculate_potential_plus(f, rho)
        for shp in SHAPES:
            if prec == native.FP64 and shp["x_radix_cap"] == 12:
                shp = dict(shp, x_radix_cap=0)
            eng.set_shape(s, **shp)
            got = eng.shape(s)
            assert got["xfwd_row_pairs"] == shp["xfwd_row_pairs"] and got["xinv_row_pairs"] == shp["xinv_row_pairs"]
            pot, et = eng.calculate_potential_plus(s, rho)
            assert np.abs(pot - pot_o).max() / np.abs(pot_o).max() < tol_pot, shp
            assert np.abs(et - et_o).max() < tol_e, shp
    finally:
        eng.slot_destroy(s)


def check_tune_caches_the_shape(eng):
    cell, f, rho_u, _ = cases.golden_case("wt_al4_displaced")
    s = cases.engine_slot(eng, f, cell)
    try:
        eng.set_input(s, rho_u)
        res = eng.tune(s, iters=3)
        assert res["ms_tuned"] <= res["ms_default"] + 1e-12
        assert res["shape"] == eng.shape(s)
        s2 = cases.engine_slot(eng, f, cell)
        try:
            assert eng.shape(s2) == res["shape"]
            pot_o, et_o = fn.calculate_potential_plus(f, rho_u)
            pot, et = eng.calculate_potential_plus(s2, rho_u)
            assert np.abs(et - et_o).max() < 1e-10
        finally:
            eng.slot_destroy(s2)
    finally:
        eng.slot_destroy(s)


def test_shapes_same_results(emu_engine):
    check_shapes_same_results(emu_engine)


def test_shapes_same_results_wgc(emu_engine):
    check_shapes_same_results(emu_engine, "wgc_al4_fcc")


def test_shapes_same_results_fp32(emu_engine):
    check_shapes_same_results(emu_engine, "wgc_al4_fcc", prec=native.FP32, tol_pot=1e-5, tol_e=2e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wt_al4_displaced", "wgc_al4_fcc"])
def test_shapes_same_results_on_gpu(gpu_engine, name):
    check_shapes_same_results(gpu_engine, name)
    check_shapes_same_results(gpu_engine, name, prec=native.FP32, tol_pot=1e-5, tol_e=2e-5)


@pytest.mark.gpu
def test_tune_caches_the_shape_on_gpu(gpu_engine):
    check_tune_caches_the_shape(gpu_engine)


def test_tune_caches_the_shape(emu_engine):
    check_tune_caches_the_shape(emu_engine)


def test_shape_out_of_range(emu_engine):
    cell, f, _, _ = cases.golden_case("wt_al4_displaced")
    s = cases.engine_slot(emu_engine, f, cell)
    try:
        for bad in (dict(x_radix_cap=7, xfwd_row_pairs=1, xinv_row_pairs=1),
                    dict(x_radix_cap=0, xfwd_row_pairs=0, xinv_row_pairs=1),
                    dict(x_radix_cap=0, xfwd_row_pairs=1, xinv_row_pairs=33),
                    dict(x_radix_cap=0, xfwd_row_pairs=1, xinv_row_pairs=1, yz_threads=128)):
            with pytest.raises(native.OfdftError):
                emu_engine.set_shape(s, **bad)
    finally:
        emu_engine.slot_destroy(s)
