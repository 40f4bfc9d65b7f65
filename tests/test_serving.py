"""Serving scheduler logic on the host-emulation engine (CPU): admission by
device footprint, continuous batching, the FP32 -> FP64 hand-off, and that a
request's result is the same alone and in the mix."""
import numpy as np
import pytest

from profess_b200 import serving, workloads as wl


def small_cell(seed, kinetic=4):
    c = wl.fcc_al((1, 1, 1), sigma_ang=0.05, grid=(16, 16, 16), seed=seed, kinetic=kinetic)
    if kinetic == 5:
        import math
        c.alpha, c.beta = (5 + math.sqrt(5)) / 6, (5 - math.sqrt(5)) / 6
    return c


def test_partition_is_disjoint_and_complete():
    rids = list(range(37))
    parts = [serving.partition(rids, r, 4) for r in range(4)]
    assert sorted(sum(parts, [])) == rids
    assert all(set(a).isdisjoint(b) for i, a in enumerate(parts) for b in parts[i + 1:])


def _run(eng, reqs, budget):
    srv = serving.Server(eng, hbm_budget=budget, max_active=8, ticks_per_poll=4)
    for r in reqs:
        srv.submit(r)
    return {r.rid: r for r in srv.run_until_done(timeout=600)}


def test_results_same_alone_and_in_the_mix(emu_engine):
    reqs = [serving.Request(rid=i, cell=small_cell(i, kinetic=4 if i != 2 else 5), arrival=0.0,
                            mode=serving.MODE_MIXED if i % 2 == 0 else serving.MODE_FP64, pot_tol=1e-6, seed=i)
            for i in range(4)]
    mix = _run(emu_engine, reqs, budget=10 ** 12)
    assert sorted(mix) == [0, 1, 2, 3]
    for r in reqs:
        alone = _run(emu_engine, [r], budget=10 ** 12)[r.rid]
        assert np.array_equal(alone.energy, mix[r.rid].energy)
        assert alone.stats["num_evals"] == mix[r.rid].stats["num_evals"]


def test_admission_respects_the_budget(emu_engine):
    reqs = [serving.Request(rid=i, cell=small_cell(10 + i), arrival=0.0, mode=serving.MODE_FP64, seed=i)
            for i in range(3)]
    one = serving.footprint(emu_engine.lib, reqs[0].cell, serving.MODE_FP64)
    srv = serving.Server(emu_engine, hbm_budget=int(1.5 * one), max_active=8, ticks_per_poll=4)
    for r in reqs:
        srv.submit(r)
    peak = 0
    while srv.future or srv.waiting or srv.active:
        srv.step()
        peak = max(peak, len(srv.active))
        assert srv.used <= srv.budget
    assert peak == 1 and len(srv.results) == 3
    stats = serving.latency_stats(srv.results)
    assert stats["solves"] == 3 and stats["p99_s"] >= stats["p50_s"] > 0


def test_oversize_request_is_rejected(emu_engine):
    r = serving.Request(rid=0, cell=small_cell(1), arrival=0.0, mode=serving.MODE_FP64)
    srv = serving.Server(emu_engine, hbm_budget=1000)
    srv.submit(r)
    with pytest.raises(ValueError):
        srv.step()
