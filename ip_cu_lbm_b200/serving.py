"""Continuous-batching serving of many simulations on one GPU.

Requests (a 2-D or 3-D case and a step count) arrive over time. The server
admits them first-in first-out while the device memory they need fits the
HBM budget, keeps every admitted simulation resident, and advances all of
them together. Each tick is one batched call (ipcu_batch_launch_each) that
takes every 2-D simulation to its own end of the tick with one launch per
step for every kernel class, CTAs of a persistent grid walking a device work
list of (simulation, tile); the tick's launches are captured into one CUDA
graph and replayed (the executable graph updated in place while the batch
keeps its shape), and the grid of each kernel class is chosen by the
Autotuner. 3-D simulations replay their own step graphs on their own streams
beside the batch. Finished simulations are retired at the tick boundary --
their results copied into pooled pinned buffers on their own streams, handed
out on a worker thread a tick later, their memory freed -- and waiting
requests admitted into the space: requests that arrive while others are on
the GPU join the running batch.

A simulation's arithmetic is the single-run kernel's, tile by tile, so its
result is the same alone and in any mix.
"""
from __future__ import annotations

import ctypes
import heapq
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .sim import Sim
from .sim3d import Sim3D


def new_stream():
    """A dedicated non-blocking CUDA stream (ipcu_stream_create), as an int handle."""
    h = ctypes.c_void_p()
    _lib.check(_lib.lib().ipcu_stream_create(ctypes.byref(h)), "ipcu_stream_create")
    return h.value


class Batch:
    """Owner of an ipcu_batch (device parameter array and work list)."""

    def __init__(self, stream=None):
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().ipcu_batch_create(stream, ctypes.byref(h)), "ipcu_batch_create")
        self._h = h

    def step(self, sims, n):
        """Advances `sims` by n steps and waits."""
        if not sims or n <= 0:
            return
        arr = (ctypes.c_void_p * len(sims))(*[s._h.value for s in sims])
        _lib.check(_lib.lib().ipcu_batch_step(self._h, arr, len(sims), int(n)), "ipcu_batch_step")

    def launch(self, sims, n):
        """Enqueues n steps of `sims` without waiting (each simulation's own
        stream is ordered after them)."""
        if not sims or n <= 0:
            return
        arr = (ctypes.c_void_p * len(sims))(*[s._h.value for s in sims])
        _lib.check(_lib.lib().ipcu_batch_launch(self._h, arr, len(sims), int(n)), "ipcu_batch_launch")

    def launch_each(self, sims, steps):
        """Enqueues steps[i] steps of sims[i] without waiting, in one call
        (ipcu_batch_launch_each): those still stepping share each launch."""
        if not sims:
            return
        arr = (ctypes.c_void_p * len(sims))(*[s._h.value for s in sims])
        cnt = (ctypes.c_int64 * len(sims))(*[int(n) for n in steps])
        _lib.check(_lib.lib().ipcu_batch_launch_each(self._h, arr, cnt, len(sims)), "ipcu_batch_launch_each")

    def sync(self):
        _lib.check(_lib.lib().ipcu_batch_sync(self._h), "ipcu_batch_sync")

    def set_graph(self, enable=True):
        """Graph mode: each launch call's kernels captured into one CUDA
        graph and replayed (ipcu_batch_set_graph; not on the legacy stream)."""
        _lib.check(_lib.lib().ipcu_batch_set_graph(self._h, 1 if enable else 0), "ipcu_batch_set_graph")

    def graph_stats(self):
        """(in-place graph updates, instantiations) so far."""
        u, i = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(_lib.lib().ipcu_batch_graph_stats(self._h, ctypes.byref(u), ctypes.byref(i)),
                   "ipcu_batch_graph_stats")
        return u.value, i.value

    def set_ctas(self, kernel_class, ctas_per_sm):
        """CTAs per SM of the batched grid for a kernel class (Sim.kernel_class);
        0 restores the default."""
        st, q, geo, kind = (int(v) for v in kernel_class[:4])
        _lib.check(_lib.lib().ipcu_batch_set_ctas(self._h, st, q, geo, kind, int(ctas_per_sm)), "ipcu_batch_set_ctas")

    def mark(self):
        """Handle of the point reached by everything enqueued so far."""
        m = _lib.lib().ipcu_batch_mark(self._h)
        if m < 0:
            _lib.check(m, "ipcu_batch_mark")
        return m

    def wait_mark(self, m):
        _lib.check(_lib.lib().ipcu_batch_wait_mark(self._h, int(m)), "ipcu_batch_wait_mark")

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
    body: dict = field(default=None, compare=False)  # Sim.attach_ellipse arguments (immersed body)
    ny: int = field(default=0, compare=False)  # > 0: a 3-D request (Sim3D, nx x ny x nz)
    stream: object = field(default=None, compare=False, repr=False)  # the simulation's own CUDA stream
    # filled by the server
    sim: object = field(default=None, compare=False, repr=False)
    remaining: int = field(default=0, compare=False)
    admitted: float = field(default=None, compare=False)
    finished: float = field(default=None, compare=False)
    result: dict = field(default=None, compare=False, repr=False)

    @property
    def cells(self):
        return self.nx * self.nz * (self.ny if self.ny else 1)

    @property
    def is3d(self):
        return self.ny > 0


def request_bytes(req: Request) -> int:
    """Device bytes a request needs once admitted (same formula as
    ipcu_sim_device_bytes; 3-D: two buffers of f, g, the FP32 force planes
    and, with 16-bit storage, the reference planes, as
    ipcu_sim3d_bytes_per_cell counts them)."""
    if req.is3d:  # (a sphere adds its force density and about 4 MB of update scratch)
        per_cell = 232 if req.kwargs.get("storage", "f32") == "f32" else 148
        return per_cell * req.cells + ((12 * req.cells + (4 << 20)) if req.body is not None else 0)
    f32 = req.kwargs.get("storage", "f32") == "f32"
    esz, nmac = (4, 3) if f32 else (2, 4)  # 16-bit storage keeps p* in a 4th FP32 plane
    pf = req.kwargs.get("scalar", "salinity") == "phase"
    if pf:
        nmac += 2  # previous step's phi u, phi w
    q = max(req.kwargs.get("q_scalar", 5), 1)
    N = req.cells
    ib = 0
    if req.body is not None:  # force density, tile flags, markers, body state
        ib = 8 * N + ((req.nx + 31) // 32) * ((req.nz + 15) // 16) + 40 * req.body.get("markers", 240) + 104
    return (2 * (esz * (9 + q) * N + 4 * nmac * N) + 4 * (3 * (req.nx + req.nz) + 10 * max(req.nx, req.nz)) + 2048
            + (4 * (req.nx + req.nz) if pf else 0) + ib)


def make_sim(req: Request, stream=None):
    """The request's simulation (2-D Sim with its body, or Sim3D)."""
    if req.is3d:
        s = Sim3D(req.nx, req.ny, req.nz, s0=req.s0, stream=stream, **req.kwargs)
        if req.body is not None:
            s.attach_sphere(**req.body)
        return s
    s = Sim(req.nx, req.nz, s0=req.s0, stream=stream, **req.kwargs)
    if req.body is not None:
        s.attach_ellipse(**req.body)
    return s


def kernel_class(req: Request):
    """Batched-kernel class of a 2-D request: (storage, scalar lattice,
    geometry, scalar kind, has a body)."""
    from .sim import GEOMETRY, SCALAR, STORAGE

    kw = req.kwargs
    return (STORAGE[kw.get("storage", "f32")], int(kw.get("q_scalar", 5)), GEOMETRY[kw.get("geometry", "uniform")],
            SCALAR[kw.get("scalar", "salinity")], req.body is not None)


class Autotuner:
    """Chooses the batched grid per kernel class by measurement: for each
    class (storage, scalar lattice, geometry, scalar kind, body) it runs a
    sample of that class's requests together in a private batch, times
    `steps` batched steps for each candidate number of CTAs per SM (the
    persistent grid walks the tile work list), and keeps the fastest.
    Choices are cached per class (and can be saved and reloaded as JSON).
    The tile (32 x 16 cells, 256 threads, 2 cells per thread) is fixed at
    compile time, so the grid is what is tuned at run time."""

    def __init__(self, candidates=(1, 2, 3, 4), steps=30, sample=8, cache=None):
        self.candidates = tuple(candidates)
        self.steps = int(steps)
        self.sample = int(sample)
        self.choice = dict(cache or {})
        self.timings = {}

    @staticmethod
    def _key(cls):
        return ",".join(str(int(v)) for v in cls)

    def tune(self, requests):
        """Tunes every class present in `requests` not tuned yet; returns
        {class key: CTAs per SM}."""
        import torch

        by = {}
        for r in requests:
            if not r.is3d:
                by.setdefault(self._key(kernel_class(r)), []).append(r)
        stream = new_stream()
        try:
            for key, rs in by.items():
                if key in self.choice:
                    continue
                rs = sorted(rs, key=lambda r: r.cells)
                pick = [rs[int(i)] for i in np.linspace(0, len(rs) - 1, min(self.sample, len(rs)))]
                sims = [make_sim(r) for r in pick]
                b = Batch(stream)
                cls = sims[0].kernel_class
                times = {}
                try:
                    b.step(sims, 2)  # kernel attributes, first-touch
                    for c in self.candidates:
                        b.set_ctas(cls, c)
                        b.step(sims, 2)
                        t0 = time.perf_counter()
                        b.step(sims, self.steps)
                        times[c] = time.perf_counter() - t0
                finally:
                    b.close()
                    for s in sims:
                        s.close()
                self.choice[key] = min(times, key=times.get)
                cells = sum(s_.cells for s_ in pick)
                self.timings[key] = {c: round(cells * self.steps / t / 1e6, 1) for c, t in times.items()}
                torch.cuda.synchronize()
        finally:
            _lib.lib().ipcu_stream_destroy(stream)
        return dict(self.choice)

    def apply(self, batch):
        for key, c in self.choice.items():
            cls = tuple(int(v) for v in key.split(","))
            batch.set_ctas(cls[:4], c)

    def save(self, path):
        import json

        with open(path, "w") as f:
            json.dump({"choice": self.choice, "mlups": self.timings}, f, indent=1)

    @classmethod
    def load(cls, path, **kw):
        import json

        with open(path) as f:
            return cls(cache=json.load(f)["choice"], **kw)


class _PinnedPool:
    """Pinned host buffers by size, reused across retirements (pinned
    allocation costs milliseconds)."""

    def __init__(self):
        self.free = {}

    def get(self, n):
        import torch

        lst = self.free.get(n)
        return lst.pop() if lst else torch.empty(n, dtype=torch.float32, pin_memory=True)

    def put(self, buf):
        self.free.setdefault(buf.numel(), []).append(buf)


class Server:
    def __init__(self, budget_bytes=150e9, tick_steps=200, keep_results=("S", "ux", "uz"), stream=None,
                 admit_per_tick=64, graph=True, autotuner=None, retire_worker=True):
        """keep_results: macroscopic planes copied back per finished request
        ("S", "ux", "uz"; "p" too with 16-bit storage; 3-D requests return
        S, ux, uy, uz). stream: the batch's CUDA stream handle (default: a
        new non-blocking stream). Every admitted simulation gets a
        non-blocking stream of its own, so that its set-up (which
        synchronises that stream) never waits for the batch in flight.
        admit_per_tick bounds the set-ups done between two launches, so the
        GPU starts on the first requests while the host sets up the next
        ones. graph: each tick's batched launches are captured into one CUDA
        graph and replayed. autotuner: an Autotuner whose per-class grid
        choices the batch uses (tuned on the stream's requests at run()).
        retire_worker: finished requests are handed out (their copies
        awaited, simulations released) on a worker thread while the main
        thread launches and admits."""
        from concurrent.futures import ThreadPoolExecutor

        self.admit_per_tick = int(admit_per_tick)
        self._own_stream = None
        if stream is None:
            self._own_stream = new_stream()
            stream = self._own_stream
        self.budget = float(budget_bytes)
        self.tick_steps = int(tick_steps)
        self.keep = keep_results
        self.stream = stream
        self.batch = Batch(stream)
        if graph:
            self.batch.set_graph(True)
        self.autotuner = autotuner
        if autotuner is not None:
            autotuner.apply(self.batch)
        self.pool = _PinnedPool()
        self.worker = ThreadPoolExecutor(max_workers=1) if retire_worker else None
        self.pending_retire = None  # the worker's current job: (future, bytes it frees)
        self.waiting: list[Request] = []
        self.active: list[Request] = []
        self.done: list[Request] = []
        self.in_use = 0
        self.cell_updates = 0
        self.t_admit = self.t_step = self.t_retire = 0.0  # host seconds per phase (main thread)
        self.t_retire_worker = 0.0  # seconds the worker spent handing out results
        self.retiring = []      # finished requests whose results are being copied back
        self.prev_mark = None   # progress mark of the previous tick's batch

    def submit(self, req: Request, now: float):
        req.remaining = req.steps
        heapq.heappush(self.waiting, req)

    def _admit(self, now):
        t0 = time.perf_counter()
        admitted = 0
        while (self.waiting and admitted < self.admit_per_tick
               and self.in_use + request_bytes(self.waiting[0]) <= self.budget):
            admitted += 1
            r = heapq.heappop(self.waiting)
            r.stream = new_stream()
            r.sim = make_sim(r, r.stream)
            r.admitted = now
            self.in_use += request_bytes(r)
            self.active.append(r)
        self.t_admit += time.perf_counter() - t0

    def _collect_retired(self, wait):
        """Applies the worker's finished job (memory it freed)."""
        if self.pending_retire is None:
            return
        fut, nbytes = self.pending_retire
        if not wait and not fut.done():
            return
        fut.result()
        self.in_use -= nbytes
        self.pending_retire = None

    def tick(self, clock):
        """One pipelined tick: enqueue up to tick_steps for every active
        simulation (2-D: one batched call; 3-D: graph replays on their own
        streams, which overlap the batch), enqueue the result copies of
        those that finish with it, then -- while the GPU runs -- hand the
        previous tick's finishers to the retire worker, admit waiting
        requests, and wait for the previous tick's batch, so the host stays
        one tick ahead of the GPU."""
        if not self.active and not self.retiring:
            self._collect_retired(wait=True)
            self._admit(clock())
            if not self.active:
                return 0
        t0 = time.perf_counter()
        two = [r for r in self.active if not r.is3d]
        steps = [min(self.tick_steps, r.remaining) for r in two]
        self.batch.launch_each([r.sim for r in two], steps)
        for r in self.active:
            n = min(self.tick_steps, r.remaining)
            if r.is3d:
                r.sim.step_graph(n)
            r.remaining -= n
            self.cell_updates += r.cells * n
        mark = self.batch.mark()
        # finishers: copy the macroscopic planes back on their own streams,
        # which the batch launch ordered after their last steps
        still, new_retiring = [], []
        for r in self.active:
            if r.remaining == 0:
                if r.is3d:
                    buf = self.pool.get(4 * r.cells)
                    r.sim.macro_async(buf)
                else:
                    buf = self.pool.get(r.sim.mac_planes() * r.cells)
                    r.sim.download(None, None, buf)
                new_retiring.append((r, buf))
            else:
                still.append(r)
        self.active = still
        t1 = time.perf_counter()
        self._retire(self.retiring, clock)
        self.retiring = new_retiring
        t2 = time.perf_counter()
        a0 = self.t_admit
        self._collect_retired(wait=False)
        self._admit(clock())
        if self.prev_mark is not None:
            self.batch.wait_mark(self.prev_mark)
        self.prev_mark = mark
        t3 = time.perf_counter()
        self.t_retire += t2 - t1
        self.t_step += (t1 - t0) + (t3 - t2) - (self.t_admit - a0)
        if not self.active and not self.waiting:
            # drain: the last batch and its finishers
            self.batch.wait_mark(mark)
            self._retire(self.retiring, clock)
            self.retiring = []
            self._collect_retired(wait=True)
            self.prev_mark = None
        return len(self.active) + len(self.retiring)

    def _retire(self, retiring, clock):
        """Hands the requests whose copies were enqueued a tick ago to the
        worker (or retires them here without one)."""
        if not retiring:
            return
        self._collect_retired(wait=True)  # one job at a time: done list and pool stay ordered
        nbytes = sum(request_bytes(r) for r, _ in retiring)
        if self.worker is None:
            self._finish(retiring, clock)
            self.in_use -= nbytes
        else:
            self.pending_retire = (self.worker.submit(self._finish, retiring, clock), nbytes)

    def _finish(self, retiring, clock):
        """Results of requests whose copies were enqueued a tick ago: wait
        for each copy, keep the planes (copied out of the pooled pinned
        buffer), release the simulation (stream-ordered)."""
        t0 = time.perf_counter()
        for r, buf in retiring:
            r.sim.sync()
            a = buf.numpy()
            if r.is3d:
                shape = (r.nz, r.ny, r.nx)
                r.result = {k: a[i * r.cells:(i + 1) * r.cells].reshape(shape).copy()
                            for i, k in enumerate(("S", "ux", "uy", "uz"))}
                if r.body is not None:
                    r.result["body"] = r.sim.body()
            else:
                planes = {"S": 0, "ux": 1, "uz": 2, "p": 3}
                r.result = {k: a[planes[k] * r.cells:(planes[k] + 1) * r.cells].reshape(r.nz, r.nx).copy()
                            for k in self.keep}
                if r.body is not None:
                    r.result["body"] = r.sim.body()
            self.pool.put(buf)
            r.finished = clock()
            r.sim.close()
            r.sim = None
            _lib.lib().ipcu_stream_destroy(r.stream)  # the frees queued on it still run
            r.stream = None
            self.done.append(r)
        self.t_retire_worker += time.perf_counter() - t0

    def run(self, requests, clock=time.perf_counter):
        """Serve `requests` (arrival times relative to the start); returns stats."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        rel = lambda: clock() - t0
        i = 0
        while i < len(pending) or self.waiting or self.active or self.retiring or self.pending_retire:
            now = rel()
            while i < len(pending) and pending[i].arrival <= now:
                self.submit(pending[i], now)
                i += 1
            if not self.waiting and not self.active and not self.retiring:
                self._collect_retired(wait=True)
                if i < len(pending):
                    time.sleep(max(0.0, min(pending[i].arrival - now, 0.05)))
                continue
            self.tick(rel)
        wall = rel()
        lat = np.array([r.finished - r.arrival for r in self.done])
        upd, inst = self.batch.graph_stats()
        return {"requests": len(self.done), "wall_s": wall, "cell_updates": self.cell_updates,
                "mlups": self.cell_updates / wall / 1e6,
                "host_s": {"admit": round(self.t_admit, 4), "step": round(self.t_step, 4),
                           "retire": round(self.t_retire, 4), "retire_worker": round(self.t_retire_worker, 4)},
                "graph": {"updates": upd, "instantiations": inst},
                "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None}

    def close(self):
        self.batch.sync()
        self._collect_retired(wait=True)
        for r in self.active + [r for r, _ in self.retiring]:
            if r.sim is not None:
                r.sim.sync()
                r.sim.close()
                r.sim = None
            if r.stream is not None:
                _lib.lib().ipcu_stream_destroy(r.stream)
                r.stream = None
        if self.worker is not None:
            self.worker.shutdown(wait=True)
        self.batch.close()
        if self._own_stream is not None:
            _lib.lib().ipcu_stream_destroy(self._own_stream)
            self._own_stream = None


def lock_exchange_request(rid, nx, nz, steps, arrival=0.0, storage="f16", seed=0):
    """A 2-D lock-exchange request: S = 1 on the left half (seeded interface
    noise), D2Q9 MRT + D2Q5, uniform grid, bounce-back, lattice units. The
    reduced gravity g' = 1e-4 (64 / nz) keeps the front speed, about
    sqrt(g' nz) / 2, at 0.04 lattice units on every grid height."""
    rng = np.random.default_rng(seed)
    S0 = np.where(np.arange(nx)[None, :] < nx // 2, 1.0, 0.0) * np.ones((nz, 1))
    S0[:, nx // 2 - 1: nx // 2 + 1] += rng.uniform(-1e-4, 1e-4, (nz, 2))
    gp = 1e-4 * 64.0 / nz
    kw = dict(q_scalar=5, geometry="uniform", storage=storage, wall="bb", mrt=True, tau=0.53, taus=0.503,
              rho_sal=gp, g_bouss=gp)
    return Request(arrival=arrival, rid=rid, nx=nx, nz=nz, steps=steps, kwargs=kw, s0=S0.ravel())


def falling_ellipse_request(rid, nx, nz, steps, arrival=0.0, storage="f16", seed=0):
    """A 2-D settling-ellipse request after the immersed-boundary case,
    scaled to the grid: semi-axes a = max(nx/40, 8), b = a/2 (20 x 10 on an
    800-wide box; the coupling needs b >= 4 cells at this density ratio, a
    body thinner than that lies wholly inside its own Peskin stencils and
    its interior fluid no longer moves with it), markers at about 2.5 per
    unit arc length (48..512), density ratio 1.1, tilt 45 degrees, released
    from rest at (nx/2, 0.85 nz) with a seeded +-2 % jitter; gravity
    1e-5 (20/a)^2 keeps the settling speed comparable across sizes; D2Q9
    MRT, nu = 0.02, bounce-back, no scalar, lattice units."""
    rng = np.random.default_rng(seed)
    a = max(nx / 40.0, 8.0)
    b = a / 2.0
    per = np.pi * (3 * (a + b) - np.sqrt((3 * a + b) * (a + 3 * b)))
    markers = int(min(max(round(2.5 * per), 48), 512))
    j = 1.0 + rng.uniform(-0.02, 0.02, 2)
    kw = dict(q_scalar=0, geometry="uniform", storage=storage, wall="bb", mrt=True, tau=0.56)
    body = dict(xc=nx / 2 * j[0], zc=0.85 * nz * j[1], a=a, b=b, markers=markers, theta=np.pi / 4, rho_s=1.1,
                rho_f=1.0, gravity=1e-5 * (20.0 / a) ** 2, iters=3)
    return Request(arrival=arrival, rid=rid, nx=nx, nz=nz, steps=steps, kwargs=kw, s0=np.zeros(nx * nz), body=body)


def rayleigh_taylor_request(rid, nx, nz, steps, arrival=0.0, storage="f16", seed=0):
    """A 2-D Rayleigh-Taylor request on the conservative Allen-Cahn phase
    field: heavy fluid (phi = 1, density 3) over light (phi = 0, density 1),
    interface width W = 4, mobility (tau_phi - 1/2)/3 = 0.02, a seeded
    single-mode perturbation of amplitude 0.05 nx, slip walls, D2Q9 MRT with
    a D2Q9 phase lattice, lattice units. Gravity g = 1e-5 (256 / nx) keeps
    the growth speed sqrt(At g nx) near 0.04 on every grid width."""
    rng = np.random.default_rng(seed)
    xx, zz = np.meshgrid(np.arange(nx) + 0.5, np.arange(nz) + 0.5)
    amp = 0.05 * nx * (1.0 + rng.uniform(-0.02, 0.02))
    zi = nz / 2 + amp * np.cos(2 * np.pi * xx / nx + rng.uniform(0, 2 * np.pi))
    phi0 = 0.5 * (1.0 + np.tanh(2.0 * (zz - zi) / 4.0))
    kw = dict(q_scalar=9, geometry="uniform", storage=storage, wall="slip", mrt=True, tau=0.56, taus=0.56,
              scalar="phase", rhoL=1.0, rhoH=3.0, sigma=5e-5, pf_width=4.0, gravity=1e-5 * 256.0 / nx)
    return Request(arrival=arrival, rid=rid, nx=nx, nz=nz, steps=steps, kwargs=kw, s0=phi0.ravel())


def stratified_box_request(rid, nx, ny, nz, steps, arrival=0.0, seed=0, sphere=True, storage="f32"):
    """A 3-D falling-sphere request after the sphere configuration: D3Q19
    MRT + D3Q7 salinity with a linear stratification S = 1 - z/H (seeded
    1e-4 noise), Boussinesq g' = 1e-5, rho = 1 + 1e-3 S, tau = 0.55, tau_s =
    0.52, bounce-back walls, uniform grid, FP32 storage by default (the 3-D
    kernel is issue-bound: 16-bit storage saves memory, not time), and a
    sphere of diameter nx/8 (radius at least 4 cells)
    with markers at about one per unit area, density ratio 1.5, released from
    rest at 0.8 of the height with a seeded lateral offset of at most one
    cell, gravity 2e-5 (sphere=False: the stratified box alone)."""
    rng = np.random.default_rng(seed)
    zz = np.broadcast_to((np.arange(nz) + 0.5)[:, None, None] / nz, (nz, ny, nx))
    S0 = 1.0 - zz + 1e-4 * rng.uniform(-1, 1, (nz, ny, nx))
    kw = dict(tau=0.55, taus=0.52, rho_sal=1e-3, g_bouss=1e-5)
    if storage != "f32":
        kw["storage"] = storage
    body = None
    if sphere:
        off = rng.uniform(-1.0, 1.0, 2)
        body = dict(xc=nx / 2 + off[0], yc=ny / 2 + off[1], zc=0.8 * nz, radius=max(nx / 16.0, 4.0), rho_s=1.5,
                    rho_f=1.0, gravity=2e-5, iters=3)
    return Request(arrival=arrival, rid=rid, nx=nx, nz=nz, ny=ny, steps=steps, kwargs=kw, s0=S0.ravel(), body=body)
