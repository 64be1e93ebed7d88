"""Continuous-batching serving of many simulations on one GPU.

Requests (a 2-D case and a step count) arrive over time. The server admits
them first-in first-out while the device memory they need fits the HBM
budget, keeps every admitted simulation resident, and advances all of them
together: each tick is one batched call (ipcu_batch_step) that runs one launch
per step for every kernel class, CTAs walking a device work list of
(simulation, tile). Finished simulations are retired at the tick boundary,
their memory freed, and waiting requests admitted into the space -- requests
that arrive while others are on the GPU join the running batch.

A simulation's arithmetic is the single-run kernel's, tile by tile, so its
result is the same alone and in any mix.
"""
from __future__ import annotations

import ctypes
import heapq
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .sim import Sim


class Batch:
    """Owner of an ipcu_batch (device parameter array and work list)."""

    def __init__(self, stream=None):
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().ipcu_batch_create(stream, ctypes.byref(h)), "ipcu_batch_create")
        self._h = h

    def step(self, sims, n):
        if not sims or n <= 0:
            return
        arr = (ctypes.c_void_p * len(sims))(*[s._h.value for s in sims])
        _lib.check(_lib.lib().ipcu_batch_step(self._h, arr, len(sims), int(n)), "ipcu_batch_step")

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().ipcu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass(order=True)
class Request:
    arrival: float
    rid: int = field(compare=False)
    nx: int = field(compare=False)
    nz: int = field(compare=False)
    steps: int = field(compare=False)
    kwargs: dict = field(default_factory=dict, compare=False)
    s0: np.ndarray = field(default=None, compare=False)
    # filled by the server
    sim: Sim = field(default=None, compare=False, repr=False)
    remaining: int = field(default=0, compare=False)
    admitted: float = field(default=None, compare=False)
    finished: float = field(default=None, compare=False)
    result: dict = field(default=None, compare=False, repr=False)

    @property
    def cells(self):
        return self.nx * self.nz


def request_bytes(req: Request) -> int:
    """Device bytes a request needs once admitted (same formula as ipcu_sim_device_bytes)."""
    esz = 4 if req.kwargs.get("storage", "f32") == "f32" else 2
    q = max(req.kwargs.get("q_scalar", 5), 1)
    N = req.cells
    return 2 * (esz * (9 + q) * N + 12 * N) + 4 * (3 * (req.nx + req.nz) + 10 * max(req.nx, req.nz)) + 2048


class Server:
    def __init__(self, budget_bytes=150e9, tick_steps=200, keep_results=("S", "ux", "uz"), stream=None):
        self.budget = float(budget_bytes)
        self.tick_steps = int(tick_steps)
        self.keep = keep_results
        self.stream = stream
        self.batch = Batch(stream)
        self.waiting: list[Request] = []
        self.active: list[Request] = []
        self.done: list[Request] = []
        self.in_use = 0
        self.cell_updates = 0

    def submit(self, req: Request, now: float):
        req.remaining = req.steps
        heapq.heappush(self.waiting, req)

    def _admit(self, now):
        while self.waiting and self.in_use + request_bytes(self.waiting[0]) <= self.budget:
            r = heapq.heappop(self.waiting)
            r.sim = Sim(r.nx, r.nz, s0=r.s0, stream=self.stream, **r.kwargs)
            r.admitted = now
            self.in_use += r.sim.device_bytes()
            self.active.append(r)

    def tick(self, clock):
        """Admit, advance every active simulation by up to tick_steps, retire."""
        self._admit(clock())
        if not self.active:
            return 0
        groups = {}
        for r in self.active:
            groups.setdefault(min(self.tick_steps, r.remaining), []).append(r)
        for n, rs in sorted(groups.items(), reverse=True):
            self.batch.step([r.sim for r in rs], n)
            for r in rs:
                r.remaining -= n
                self.cell_updates += r.cells * n
        now = clock()
        still = []
        for r in self.active:
            if r.remaining == 0:
                r.finished = now
                r.result = {k: r.sim.get(k) for k in self.keep}
                self.in_use -= r.sim.device_bytes()
                r.sim.close()
                r.sim = None
                self.done.append(r)
            else:
                still.append(r)
        self.active = still
        return len(self.active)

    def run(self, requests, clock=time.perf_counter):
        """Serve `requests` (arrival times relative to the start); returns stats."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        rel = lambda: clock() - t0
        i = 0
        while i < len(pending) or self.waiting or self.active:
            now = rel()
            while i < len(pending) and pending[i].arrival <= now:
                self.submit(pending[i], now)
                i += 1
            if not self.waiting and not self.active and i < len(pending):
                time.sleep(max(0.0, min(pending[i].arrival - now, 0.05)))
                continue
            self.tick(rel)
        wall = rel()
        lat = np.array([r.finished - r.arrival for r in self.done])
        return {"requests": len(self.done), "wall_s": wall, "cell_updates": self.cell_updates,
                "mlups": self.cell_updates / wall / 1e6,
                "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None}

    def close(self):
        for r in self.active:
            if r.sim is not None:
                r.sim.close()
        self.batch.close()


def lock_exchange_request(rid, nx, nz, steps, arrival=0.0, storage="f16", seed=0):
    """A 2-D lock-exchange request: S = 1 on the left half (seeded interface
    noise), D2Q9 MRT + D2Q5, uniform grid, bounce-back, lattice units."""
    rng = np.random.default_rng(seed)
    S0 = np.where(np.arange(nx)[None, :] < nx // 2, 1.0, 0.0) * np.ones((nz, 1))
    S0[:, nx // 2 - 1: nx // 2 + 1] += rng.uniform(-1e-4, 1e-4, (nz, 2))
    kw = dict(q_scalar=5, geometry="uniform", storage=storage, wall="bb", mrt=True, tau=0.53, taus=0.503,
              rho_sal=1e-4, g_bouss=1e-4, s_ref=0.5)
    return Request(arrival=arrival, rid=rid, nx=nx, nz=nz, steps=steps, kwargs=kw, s0=S0.ravel())
