"""Continuous-batching density-solve server on one GPU (one engine).

Requests (a cell plus solve options) arrive over time; the server admits a
waiting request when its device footprint fits the HBM budget and engine
slots are free, builds its tables on the device, and starts its solve in the
engine, where it shares every kernel launch with the solves already running.
The host-side input of a request (its initial density) is prepared by a
small thread pool as soon as it arrives, so the engine keeps running the
admitted solves meanwhile; its Ewald energy is summed on the device at
admission.
A mixed-precision request runs an FP32 slot until the FP32 line-search floor
(or the FP32 tolerance), then FP64 refinement iterations in an FP64 slot
started from the FP32 density on the device; a plain request runs FP64
throughout.  A mixed request sets up its FP64 slot at admission (kernel,
ion potential and Ewald energy built on the device) and gives its FP32 slot
the same tables by a conversion on the device, so it pays for one set-up like
a plain request; the FP32 slot is released as soon as the refinement has
taken its density.  Densities and solver state stay on the device until the
result is read.  Finished slots are released at once, so waiting requests enter as
soon as memory frees up.  Latency is arrival to result.

Multi-GPU serving runs one server per GPU (replicas); ``partition`` assigns
request ids to ranks with no exchange on the data path.
"""
from __future__ import annotations

import collections
import concurrent.futures
import contextlib
import dataclasses
import os
import time

import numpy as np

from . import native
from .cell import setup_slot, slot_like
from .workloads import Cell, initial_density

MODE_MIXED = "mixed"
MODE_FP64 = "fp64"


@dataclasses.dataclass
class Request:
    rid: int
    cell: Cell
    arrival: float = 0.0          # seconds after the server's start
    mode: str = MODE_MIXED
    fp32_tol: float = 3.0e-5
    refine_iters: int = 3
    pot_tol: float = 1.0e-6
    seed: int = 0


@dataclasses.dataclass
class Result:
    rid: int
    energy: np.ndarray
    stats: dict
    arrival: float
    admitted: float
    finished: float
    nion: int
    grid: tuple
    mode: str

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def partition(rids, rank: int, world: int):
    """Replica assignment of request ids to ranks (round robin)."""
    return [r for r in rids if r % world == rank]


def slot_bytes(lib, cell: Cell, precision) -> int:
    return native.slot_footprint(lib, cell.grid, cell.kinetic, cell.alpha, cell.beta, precision)


def footprint(lib, cell: Cell, mode: str) -> int:
    """Largest device footprint of a request: its FP64 slot, plus its FP32
    slot during the FP32 phase of a mixed request."""
    b64 = slot_bytes(lib, cell, native.FP64)
    if mode == MODE_FP64:
        return b64
    return b64 + slot_bytes(lib, cell, native.FP32)


def _pool_workers() -> int:
    return max(2, min(8, os.cpu_count() or 2))


class Server:
    def __init__(self, engine: native.Engine, hbm_budget: int, max_active: int = 24, ticks_per_poll: int = 8,
                 clock=time.perf_counter):
        self.eng = engine
        self.budget = int(hbm_budget)
        self.max_active = max_active
        self.ticks = ticks_per_poll
        self.clock = clock
        self.t0 = clock()
        self.waiting = []            # requests that have arrived, FIFO
        self.future = []             # requests not yet arrived (sorted by arrival)
        self.active = {}             # rid -> dict(state)
        self.used = 0
        self.results = []
        self.pool = concurrent.futures.ThreadPoolExecutor(max_workers=_pool_workers())
        self.prep = {}               # rid -> future of (ion-ion energy, initial density)
        self.phase_s = collections.defaultdict(float)  # host seconds per phase of the loop

    def now(self) -> float:
        return self.clock() - self.t0

    @contextlib.contextmanager
    def _phase(self, name):
        t0 = self.clock()
        try:
            yield
        finally:
            self.phase_s[name] += self.clock() - t0

    def submit(self, req: Request):
        self.future.append(req)
        self.future.sort(key=lambda r: r.arrival)

    # ------------------------------------------------------------ admission
    @staticmethod
    def _prepare(lib, req: Request):
        return initial_density(req.cell, seed=req.seed)

    def _arrivals(self):
        t = self.now()
        while self.future and self.future[0].arrival <= t:
            req = self.future.pop(0)
            self.waiting.append(req)
            self.prep[req.rid] = self.pool.submit(self._prepare, self.eng.lib, req)

    def _admit(self):
        while self.waiting and len(self.active) < self.max_active:
            req = self.waiting[0]
            b64 = slot_bytes(self.eng.lib, req.cell, native.FP64)
            b32 = slot_bytes(self.eng.lib, req.cell, native.FP32) if req.mode == MODE_MIXED else 0
            if b64 + b32 > self.budget:
                raise ValueError("request %d needs %d bytes, more than the whole budget" % (req.rid, b64 + b32))
            if self.used + b64 + b32 > self.budget:
                return
            fut = self.prep[req.rid]
            if not fut.done() and self.active:
                return  # its inputs are still being prepared; keep serving the others
            self.waiting.pop(0)
            t_adm = self.now()
            rho0 = fut.result()
            del self.prep[req.rid]
            st = {"req": req, "admitted": t_adm, "phase": None, "s32": None, "s64": None, "b64": b64, "b32": b32,
                  "fp32_stats": None}
            with self._phase("setup"):
                st["s64"] = setup_slot(self.eng, req.cell, native.FP64)  # Ewald summed on the device
                if req.mode == MODE_MIXED:
                    st["s32"] = slot_like(self.eng, req.cell, st["s64"], native.FP32)
            with self._phase("start"):
                if req.mode == MODE_FP64:
                    self.eng.start_solve(st["s64"], rho0, native.ntn_options(
                        conv_check=native.CONV_POT, pot_tol=req.pot_tol, max_iter=300))
                    st["phase"] = "fp64"
                else:
                    self.eng.start_solve(st["s32"], rho0, native.ntn_options(
                        conv_check=native.CONV_POT, pot_tol=req.fp32_tol, max_iter=300, stall_line=6))
                    st["phase"] = "fp32"
            self.used += b64 + b32
            self.active[req.rid] = st

    # ------------------------------------------------------------ progress
    def _advance(self):
        for rid in list(self.active):
            st = self.active[rid]
            req = st["req"]
            if st["phase"] == "fp32" and self.eng.poll(st["s32"]):
                # refinement in the FP64 slot from the FP32 density, on the device
                with self._phase("start"):
                    self.eng.start_solve_from_slot(st["s64"], st["s32"], native.ntn_options(
                        conv_check=native.CONV_POT, pot_tol=req.pot_tol, max_iter=req.refine_iters, stall_line=6))
                with self._phase("result"):
                    _, _, st["fp32_stats"] = self.eng.result(st["s32"], want_rho=False)
                with self._phase("release"):
                    self.eng.slot_destroy(st["s32"])
                st["s32"] = None
                self.used -= st["b32"]
                st["phase"] = "refine"
            elif st["phase"] in ("refine", "fp64") and self.eng.poll(st["s64"]):
                with self._phase("result"):
                    _, e, stats = self.eng.result(st["s64"], want_rho=False)
                if st["fp32_stats"] is not None:
                    s32 = st["fp32_stats"]
                    stats = dict(stats, fp32_evals=s32["num_evals"], fp32_outcome=s32["outcome"])
                self.results.append(Result(rid, e.copy(), stats, req.arrival, st["admitted"], self.now(),
                                           req.cell.nion, req.cell.grid, req.mode))
                with self._phase("release"):
                    self.eng.slot_destroy(st["s64"])
                self.used -= st["b64"]
                del self.active[rid]

    def step(self):
        """Admit arrived requests, run the engine for one poll interval, retire finished phases."""
        self._arrivals()
        self._admit()
        if self.active:
            with self._phase("run"):
                self.eng.run(self.ticks)
            self._advance()
            self._admit()

    def run_until_done(self, timeout: float = 3600.0):
        try:
            while self.future or self.waiting or self.active:
                if self.now() > timeout:
                    raise TimeoutError("serving did not finish")
                if not self.active and not self.waiting and self.future:
                    time.sleep(max(0.0, min(0.01, self.future[0].arrival - self.now())))
                self.step()
        finally:
            self.pool.shutdown(wait=True)
            self.pool = concurrent.futures.ThreadPoolExecutor(max_workers=_pool_workers())
        return self.results


def latency_stats(results):
    lat = np.array([r.latency for r in results])
    if len(lat) == 0:
        return {}
    span = max(r.finished for r in results) - min(r.arrival for r in results)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "solves": len(lat), "solves_per_s": len(lat) / span if span > 0 else None}
