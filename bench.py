#!/usr/bin/env python
"""Benchmark of the per-step lattice Boltzmann path (MLUPS).

Default workload (one bench step = --inner coupled lattice Boltzmann time
steps on one resident simulation): the settling-ellipse case, an 800 x 3000
uniform D2Q9 MRT box with bounce-back walls, nu = 0.02, and a 20 x 10-cell
ellipse carried by 240 markers (density ratio 1.1, tilt 45 degrees, lattice
gravity 1e-5) released from rest; FP32 (see ip_cu_lbm_b200/workloads.py).
Its 230 MB state is far larger than L2, so the step is HBM-bound.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                    [--case ib|2d|3d] [--serving]

N > 1 runs one independent replica per GPU (torchrun, one process per GPU):
the path has no exchange step, so no data-path collective is used; the
timing is a barrier + synchronize on both sides and the max over ranks.
Between timed steps L2 is flushed by writing a 256 MiB buffer. Rank 0 prints
one JSON line.

--impl reference times the reference's own implementation of this path, its
CUDA kernel library built unmodified for sm_100a (oracle/_ref), running the
case driver's kernel chain on the same workload: for the settling ellipse the
EllipticalFall2 order (equ_f .. get_IBMGw2 .. update_IBbody) on the identical
grid, body and walls, set up with the reference's own host functions
(oracle/refcase.py); nothing of this package is loaded in that process.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

INNER = 1000
METRIC = "MLUPS"


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    def __init__(self, index):
        self.index, self.samples, self.proc = index, [], None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append((time.perf_counter(), parts))

    def window(self, t0, t1):
        """Keep the samples taken between t0 and t1 (the timed region)."""
        inside = [s for s in self.samples if t0 <= s[0] <= t1]
        self.kept = inside if inside else self.samples[-1:]

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        samples = [p for _, p in getattr(self, "kept", self.samples)]
        if not samples:
            err = ""
            if self.proc is not None and self.proc.stderr is not None:
                try:
                    err = self.proc.stderr.read()[:200]
                except Exception:
                    pass
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "error": err}
        sm = [float(s[0]) for s in samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(samples)}


def measured_traffic(args):
    """DRAM bytes per launch of the default FP32 workload's step kernel from
    the committed ncu summary (profiles/traffic.json), else None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if args.storage != "f32" or (args.inner or INNER) != INNER or not os.path.exists(p):
        return None
    d = json.load(open(p)).get("step_kernel<float,5,z3,TMA>@1024x256")
    return d["dram_bytes_per_launch"] if d else None


def traffic3d(N, stretched, storage="f32"):
    """DRAM bytes per launch of the 3-D step at N cells, scaled from the
    committed 128^3 ncu capture of the same kernel (profiles/traffic.json),
    else None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    key = {"f32": "step3s_kernel<3>@128x128x128", "f16": "step3s_kernel<3,__half>@128x128x128"}.get(storage)
    d = json.load(open(p)).get(key if stretched or storage != "f32" else "step3d_kernel@128x128x128") if key else None
    return int(d["dram_bytes_per_cell"] * N) if d else None


def traffic_ib(args, lean, push=False):
    """DRAM bytes per launch of the settling-ellipse fluid step (FP32,
    800 x 3000; the push or tile form of the lean flow-only step, or the
    full one) from the committed ncu summary (profiles/traffic.json), else
    None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if args.storage != "f32" or not os.path.exists(p):
        return None
    key = ("push_kernel@800x3000" if push else
           "step_kernel<float,0,uniform,TMA,lean>@800x3000" if lean else "step_kernel<float,0,uniform,TMA>@800x3000")
    d = json.load(open(p)).get(key)
    return d["dram_bytes_per_launch"] if d else None


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def peak_label(src):
    """Where the HBM denominator came from, for the roofline object."""
    if src == "measured":
        return "measured (MEASURED_PEAKS.json hbm_gbs)"
    return "fallback (6.65 TB/s copy bandwidth measured earlier on this hardware; MEASURED_PEAKS.json absent)"


def host_cores():
    """nproc and the CPU model of this host (lscpu), for the CPU baseline."""
    model, sockets = None, None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            k, _, v = line.partition(":")
            if k.strip() == "Model name":
                model = v.strip()
            elif k.strip() == "Socket(s)":
                sockets = v.strip()
    except (OSError, subprocess.SubprocessError):
        pass
    return {"nproc": os.cpu_count(), "model": model, "sockets": sockets}


def cpu_baseline_ib(budget_s=15.0):
    """The reference's kernels restated in C++ (oracle/ipcu_oracle.cpp, FP32,
    OpenMP over all host threads), run in the EllipticalFall2 driver order on
    the settling-ellipse workload with the reference's layout (compacted
    cells, ghosts, AoS populations): as many steps as fit in budget_s."""
    import ctypes

    from oracle import oracle as _o
    from oracle import refcase

    c, host, meta = refcase.settling_ellipse_ref()
    O = _o.oracle().lib
    O.oracle_ibm_steps_f32.argtypes = [ctypes.c_void_p] * 3
    O.oracle_ibm_steps_f32.restype = ctypes.c_int
    arrs = {k: np.ascontiguousarray(v) for k, v in host.items()}
    slots = (ctypes.c_void_p * len(_o.REF_BUFS))(*[arrs[k].ctypes.data if k in arrs else None for k in _o.REF_BUFS])
    nt = meta["nt"]
    ip = (ctypes.c_longlong * 16)(nt, 1, 1, 1, 0, 0, 1, *[len(w) for w in c["walls"]], nt, 3 * meta["markers"])
    fp = (ctypes.c_float * 2)(1.0, meta["rhoH"])
    O.oracle_ibm_steps_f32(slots, ip, fp)  # warm (first touch of every page)
    n, t0 = 0, time.perf_counter()
    while n < 200 and (n < 3 or time.perf_counter() - t0 < budget_s):
        O.oracle_ibm_steps_f32(slots, ip, fp)
        n += 1
    dt = time.perf_counter() - t0
    hc = host_cores()
    return {"value": round(meta["nc"] * n / dt / 1e6, 3), "unit": METRIC, "cores": int(O.oracle_num_threads()),
            "kind": "port", "host": hc,
            "sample": f"{n} steps of the full 800x3000 settling-ellipse workload in the reference's EllipticalFall2 "
                      "kernel order, FP32, the reference kernels restated in C++ with OpenMP "
                      "(oracle/ipcu_oracle.cpp, oracle_ibm_steps_f32)"}


def cpu_baseline_2d(params, S0, meta, budget_s=12.0):
    """The FP64 structured-grid oracle (numpy port of the path) on the C2
    workload, single host thread, bounded number of steps."""
    from ip_cu_lbm_b200.cases import d2q9_mrt
    from oracle.structured import Box

    M, Minv, S = d2q9_mrt()
    p = dict(params)
    for k in ("storage", "s_ref", "mrt"):
        p.pop(k, None)
    b = Box(meta["nx"], meta["nz"], M=M, Minv=Minv, S=S, **p)
    b.S = S0.copy()
    b.g = np.array([1 / 3] + [1 / 6] * 4)[:, None, None] * S0[None]
    b.step(1)  # warm
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s and n < 50:
        b.step(1)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": round(meta["nx"] * meta["nz"] * n / dt / 1e6, 4), "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"{n} steps of the {meta['nx']}x{meta['nz']} workload, FP64 numpy oracle (oracle/structured.py)"}


def run_ours(args):
    import torch

    from ip_cu_lbm_b200 import Sim, workloads
    from ip_cu_lbm_b200.replicas import Replicas

    R = Replicas("nccl")
    rank, world, local = R.rank, R.world, R.local
    params, S0, meta = workloads.stratified_nonuniform(storage=args.storage)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    sim = Sim(meta["nx"], meta["nz"], s0=S0.ravel(), stream=stream.cuda_stream, **params)
    N = sim.N
    inner = args.inner or INNER
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    chunk = min(inner, 200)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(local) as clk:
        time.sleep(0.3)  # let the sampler start
        for w in range(args.warmup):
            flush.fill_(float(w))
            sim.step_graph(inner, chunk=chunk)
        R.barrier()
        t_start = time.perf_counter()
        for k in range(args.steps):
            flush.fill_(float(k))  # L2 flush between timed steps (not timed)
            ev[k][0].record(stream)
            sim.step_graph(inner, chunk=chunk)
            ev[k][1].record(stream)
        R.barrier()
        clk.window(t_start, time.perf_counter())
    times = [a.elapsed_time(b) for a, b in ev]
    total_ms = R.max(sum(times))
    assert sim.status() == 0, "non-finite state"
    value = world * N * inner * args.steps / (total_ms / 1e3) / 1e6
    launch_ms = total_ms / (args.steps * inner)
    bpc = sim.bytes_per_cell()
    peak, peak_src = load_peaks()
    achieved = N * bpc / (launch_ms / 1e3) / 1e9

    # end to end through the C ABI with pinned host buffers: upload the state,
    # advance INNER steps, read S, u_x, u_z back
    esz = sim.storage_bytes()
    hdt = torch.float32 if esz == 4 else torch.float16
    hf = torch.empty(9 * N, dtype=hdt, pin_memory=True)
    hg = torch.empty(5 * N, dtype=hdt, pin_memory=True)
    hm = torch.empty(sim.mac_planes() * N, dtype=torch.float32, pin_memory=True)
    sim.download(hf, hg, hm)
    sim.sync()
    e2e_steps = max(3, args.steps)
    R.barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        sim.upload(hf, hg, hm)
        sim.step_graph(inner, chunk=chunk)
        sim.download(None, None, hm)
        sim.sync()
    R.barrier()
    e2e_s = R.max(time.perf_counter() - t0)
    e2e = world * N * inner * e2e_steps / e2e_s / 1e6

    line = {
        "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.storage == "f32" else f"{args.storage}-storage/f32",
        "data": "synthetic (seeded two-layer tanh interface)",
        "config": {"workload": f"nonuniform two-layer, {meta['nx']}x{meta['nz']} D2Q9 MRT + D2Q5, tanh-stretched z "
                               f"(ratio {meta['spacing_ratio']:.2f}), 3-point upwind flux form, bounce-back",
                   "lbm_steps_per_step": inner, "cells": N, "storage": args.storage,
                   "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MiB write) between timed steps; the 36 MB state is L2-resident within a step"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": measured_traffic(args),
                     "bytes_per_cell": bpc, "peak_source": peak_label(peak_src),
                     "note": "algorithmic bytes (each stored value read once and written once) / mean launch time; "
                             "traffic = ncu dram read+write bytes of one launch (caches flushed by ncu; the "
                             "new state stays in L2, so the writes do not reach DRAM)"},
        "e2e": {"value": round(e2e, 2), "unit": METRIC, "h2d_bytes_per_step": int(hf.numel() * hf.element_size() + hg.numel() * hg.element_size()
                                                                 + hm.numel() * 4),
                "d2h_bytes_per_step": int(hm.numel() * 4)},
        "gpu_launches": args.steps * inner,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_2d(params, S0, meta)
        except Exception as e:  # reported, not fatal
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    R.close()


def run_3d(args):
    """The 3-D path at the C4 size: 160 x 160 x 640 cells (16.4M, state
    3.8 GB > L2), x and y tanh-clustered toward the centreline (spacing ratio
    3) with the 3-point conservative flux form, z uniform (--uniform3d: the
    uniform box), D3Q19 MRT + D3Q7 salinity with a linear stratification,
    bounce-back, FP32 (--storage f16 / bf16: 16-bit population storage,
    FP32 arithmetic), and the configuration's falling sphere (diameter 16
    finest cells, 804 markers, density ratio 1.5; --no-sphere leaves it
    out). A step is --inner LBM steps (default 20), each the fluid step and
    the sphere's update, replayed from a CUDA graph; the inputs are far
    larger than L2, so no flush is needed."""
    import torch

    from ip_cu_lbm_b200 import workloads
    from ip_cu_lbm_b200.replicas import Replicas
    from ip_cu_lbm_b200.sim3d import Sim3D

    R = Replicas("nccl")
    world, local = R.world, R.local
    nx, ny, nz = (int(v) for v in args.dims.split(","))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    kw, S0 = workloads.clustered_box_3d(nx, ny, nz)
    if args.uniform3d:
        for k in ("x", "wx", "y", "wy", "ns"):
            kw.pop(k)
    sim = Sim3D(nx, ny, nz, s0=S0.ravel(), stream=stream.cuda_stream, storage=args.storage, **kw)
    sphere = None if args.no_sphere else workloads.falling_sphere_3d(kw, nx, ny, nz)
    if sphere:
        sim.attach_sphere(**sphere)
    N, inner = sim.N, args.inner or 20
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(local) as clk:
        time.sleep(0.3)
        for _ in range(args.warmup):
            sim.step_graph(inner)
        R.barrier()
        t_start = time.perf_counter()
        for k in range(args.steps):
            ev[k][0].record(stream)
            sim.step_graph(inner)
            ev[k][1].record(stream)
        R.barrier()
        clk.window(t_start, time.perf_counter())
    total_ms = R.max(sum(a.elapsed_time(b) for a, b in ev))
    assert sim.status() == 0, "non-finite state"
    value = world * N * inner * args.steps / (total_ms / 1e3) / 1e6
    launch_ms = total_ms / (args.steps * inner)
    bpc = sim.bytes_per_cell()
    peak, peak_src = load_peaks()
    achieved = N * bpc / (launch_ms / 1e3) / 1e9
    # end to end: upload the state from pinned host memory (16-bit storage:
    # the force planes), advance, read back the salinity planes (16-bit: S
    # and u, formed on the device)
    f32 = args.storage == "f32"
    hf = torch.empty(19 * N, dtype=torch.float32, pin_memory=True) if f32 else None
    hg = torch.empty(7 * N, dtype=torch.float32, pin_memory=True) if f32 else None
    hF = torch.empty(3 * N, dtype=torch.float32, pin_memory=True)
    hm = None if f32 else torch.empty(4 * N, dtype=torch.float32, pin_memory=True)
    sim.download(hf, hg, hF)
    sim.sync()
    R.barrier()
    t0 = time.perf_counter()
    for _ in range(max(3, args.steps)):
        sim.upload(hf, hg, hF)
        sim.step_graph(inner)
        if f32:
            sim.download(None, hg, None)
        else:
            sim.macro_async(hm)
        sim.sync()
    R.barrier()
    e2e = world * N * inner * max(3, args.steps) / R.max(time.perf_counter() - t0) / 1e6
    h2d = 4 * (19 + 7 + 3) * N if f32 else 4 * 3 * N
    d2h = 4 * 7 * N if f32 else 4 * 4 * N
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded linear stratification)",
        "config": {"workload": (f"3-D uniform box {nx}x{ny}x{nz} D3Q19 MRT + D3Q7, bounce-back" if args.uniform3d else
                                f"3-D box {nx}x{ny}x{nz}, x and y tanh-clustered toward the centreline (ratio 3, "
                                "3-point conservative flux form, corner transport on the xy diagonals), z uniform, "
                                "D3Q19 MRT + D3Q7 linear stratification, bounce-back") +
                               (f"; falling sphere, diameter 16 cells, 804 Fibonacci markers, density ratio 1.5, "
                                f"multi-direct forcing x3, FP64 body update (released at z = {0.8 * nz:.0f})"
                                if sphere else "; no body"),
                   "lbm_steps_per_step": inner, "cells": N, "storage": args.storage,
                   "parallelism": f"replicas x{world}",
                   "l2": f"inputs ({bpc / 2 * N / 1e9:.2f} GB) larger than L2"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": traffic3d(N, not args.uniform3d, args.storage), "bytes_per_cell": bpc,
                     "peak_source": peak_label(peak_src),
                     "traffic_note": "DRAM read+write bytes per launch from the 128^3 ncu capture (profiles/traffic.json), "
                                     "scaled by cells; it grows in proportion to the cells streamed"},
        "e2e": {"value": round(e2e, 2), "unit": METRIC,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        # the fluid step, and the sphere's update: set-up, window, (interpolate, spread) per iteration,
        # write-back, body step
        "gpu_launches": (1 + (4 + 2 * sphere["iters"] if sphere else 0)) * args.steps * inner,
        "clocks": clk.summary(),
    }
    if sphere:
        b = sim.body()
        line["body_after"] = {"X": [round(v, 6) for v in b["X"]], "U": [float(f"{v:.6e}") for v in b["U"]]}
    if R.rank == 0:
        print(json.dumps(line), flush=True)
    R.close()


def ib_config(nx=800, nz=3000):
    """The settling-ellipse workload as both arms name it (identical dicts)."""
    return {"workload": f"settling ellipse: {nx}x{nz} uniform D2Q9 MRT box, bounce-back walls, nu 0.02 (lattice "
                        "units), rigid ellipse with semi-axes 20x10 cells and 240 markers at equal arc length, "
                        "density ratio 1.1, tilt 45 deg, lattice gravity 1e-5, released from rest near "
                        "(0.5, 0.85) of the box",
            "cells": nx * nz, "storage": "f32",
            "l2": "flushed (256 MiB write) between timed steps; the state is larger than L2"}


def run_ib(args):
    """The moving-immersed-boundary case (the default bench line): an
    ellipse (20 x 10 cells, 240 markers, density ratio 1.1, tilt 45 degrees)
    settling from rest in an 800 x 3000 uniform D2Q9 MRT box, gravity 1e-5
    (the second of the sweep's four values), without the optional salinity
    stratification (N^2 = 1e-6 over 3000 cells puts a hydrostatic pressure
    range of 4.5 on the weakly compressible lattice; see
    workloads.settling_ellipse). One bench step = --inner coupled steps
    (fused fluid step + the one-CTA immersed-boundary update) replayed from
    CUDA graphs; the 230 MB FP32 state exceeds L2 and a 256 MiB flush
    separates timed steps."""
    import torch

    from ip_cu_lbm_b200 import Sim, workloads
    from ip_cu_lbm_b200.replicas import Replicas

    R = Replicas("nccl")
    world, local = R.world, R.local
    params, S0, body, meta = workloads.settling_ellipse(storage=args.storage)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    sim = Sim(meta["nx"], meta["nz"], s0=S0.ravel(), stream=stream.cuda_stream, **params)
    sim.attach_ellipse(body["xc"], body["zc"], body["a"], body["b"], markers=body["markers"], theta=body["theta"],
                       rho_s=body["rho_s"], rho_f=body["rho_f"], gravity=body["gravity"], iters=body["iters"])
    N = sim.N
    inner = args.inner if args.inner else 3000
    chunk = min(inner, 100)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(local) as clk:
        time.sleep(0.3)
        for w in range(args.warmup):
            flush.fill_(float(w))
            sim.step_graph(inner, chunk=chunk)
        R.barrier()
        t_start = time.perf_counter()
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            sim.step_graph(inner, chunk=chunk)
            ev[k][1].record(stream)
        R.barrier()
        clk.window(t_start, time.perf_counter())
    total_ms = R.max(sum(a.elapsed_time(b) for a, b in ev))
    assert sim.status() == 0, "non-finite state or body window overflow"
    value = world * N * inner * args.steps / (total_ms / 1e3) / 1e6
    step_ms = total_ms / (args.steps * inner)
    bpc = sim.bytes_per_cell()
    peak, peak_src = load_peaks()
    achieved = N * bpc / (step_ms / 1e3) / 1e9
    b = sim.body()
    # the fluid step alone: the same box without the body (same kernel, same
    # bytes), timed the same way
    fluid = Sim(meta["nx"], meta["nz"], s0=S0.ravel(), stream=stream.cuda_stream, **params)
    fev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for w in range(args.warmup):
        fluid.step_graph(inner, chunk=chunk)
    R.barrier()
    for k in range(args.steps):
        flush.fill_(float(k))
        fev[k][0].record(stream)
        fluid.step_graph(inner, chunk=chunk)
        fev[k][1].record(stream)
    R.barrier()
    fluid_ms = R.max(sum(a.elapsed_time(b) for a, b in fev))
    fluid_step_ms = fluid_ms / (args.steps * inner)
    fluid_gbs = N * bpc / (fluid_step_ms / 1e3) / 1e9
    fluid_only = {"value": round(world * N * inner * args.steps / (fluid_ms / 1e3) / 1e6, 2), "unit": METRIC,
                  "achieved_gbs": round(fluid_gbs, 1), "frac": round(fluid_gbs / peak, 4),
                  "kernel": "push form" if fluid.push() else ("lean tile form" if fluid.lean() else "full step")}
    fluid.close()
    # end to end through the C ABI: every bench step uploads the whole state
    # from pinned host memory, advances --inner steps and downloads the whole
    # state and the body (the state lives on the host between steps)
    esz = sim.storage_bytes()
    hdt = torch.float32 if esz == 4 else torch.float16
    q = params["q_scalar"]
    hf = torch.empty(9 * N, dtype=hdt, pin_memory=True)
    hg = torch.empty(max(q, 1) * N, dtype=hdt, pin_memory=True)
    hm = torch.empty(sim.mac_planes() * N, dtype=torch.float32, pin_memory=True)
    sim.download(hf, hg if q else None, hm)
    sim.sync()
    R.barrier()
    t0 = time.perf_counter()
    e2e_steps = max(3, args.steps)
    for _ in range(e2e_steps):
        sim.upload(hf, hg if q else None, hm)
        sim.step_graph(inner, chunk=chunk)
        sim.download(hf, hg if q else None, hm)
        sim.body()  # synchronises the stream
    R.barrier()
    e2e = world * N * inner * e2e_steps / R.max(time.perf_counter() - t0) / 1e6
    state_bytes = hf.numel() * esz + (hg.numel() * esz if q else 0) + hm.numel() * 4
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.storage == "f32" else f"{args.storage}-storage/f32",
        "data": "synthetic (seeded release-point jitter)",
        "config": ib_config(meta["nx"], meta["nz"]) if args.storage == "f32" else
        dict(ib_config(meta["nx"], meta["nz"]), storage=args.storage),
        "lbm_steps_per_step": inner, "parallelism": f"replicas x{world}",
        "scheme": "lean flow-only step in push form (each cell collides in registers and pushes its nine "
                  "populations; 72 B/cell, no velocity planes) + multi-direct forcing (3 iterations, Peskin-4) with "
                  "an FP64 rigid-body update, CUDA-graph replay" if sim.push() else
                  "fused collide-and-stream step (lean flow-only form: populations only, velocity planes near "
                  "the body) + multi-direct forcing (3 iterations, Peskin-4) with an FP64 rigid-body update, "
                  "CUDA-graph replay" if sim.lean() else
                  "fused collide-and-stream step + multi-direct forcing (3 iterations, Peskin-4) with an FP64 "
                  "rigid-body update, CUDA-graph replay",
        "body_after": {k: round(v, 6) for k, v in b.items() if k in ("x", "z", "w", "theta")},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic_ib(args, sim.lean(), sim.push()),
                     "bytes_per_cell": bpc, "fluid_only": fluid_only,
                     "peak_source": peak_label(peak_src),
                     "note": "fluid step's algorithmic bytes / (fluid + immersed-boundary kernel time per step); "
                             "traffic = ncu dram read+write bytes of one fluid launch"},
        "e2e": {"value": round(e2e, 2), "unit": METRIC, "h2d_bytes_per_step": int(state_bytes),
                "d2h_bytes_per_step": int(state_bytes + 72)},
        "gpu_launches": 2 * args.steps * inner, "clocks": clk.summary(),
    }
    if R.rank == 0 and world == 1 and not args.no_cpu_baseline and args.storage == "f32":
        try:
            line["cpu_baseline"] = cpu_baseline_ib()
        except Exception as e:  # reported, not fatal
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    if R.rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    R.close()


def _standalone_module(relpath, name):
    """A pure-Python file of this repository loaded as a module of its own
    (no package import, so no product library is loaded)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, relpath))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def run_reference(args):
    """The reference's CUDA kernel chain (oracle/_ref) on the bench's
    workload; rank 0 only. Nothing of ip_cu_lbm_b200 is imported or loaded."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return
    from oracle import oracle as _o

    if not _o.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libipcu_ref.so missing"}))
        return
    if args.case == "3d":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no D3Q19/D3Q7 path (3-D is D3Q27 "
                                                              "only), and 160x160x640 exceeds its 2^24 float "
                                                              "cell-count limit"}))
        return
    if args.case == "2d":
        return run_reference_2d(args)
    run_reference_ib(args)


def _ref_tensors(host, dev):
    import torch

    return {k: torch.as_tensor(np.ascontiguousarray(v), device=dev,
                               dtype=torch.float32 if np.asarray(v).dtype.kind == "f" else torch.int32)
            for k, v in host.items()}


def run_reference_ib(args):
    """The reference's EllipticalFall2 kernel chain (ref:
    EllipticalFall2/EllipticalFallxz.cu:344-430: equ_f, Force, col_f_MRT,
    IP_process, update_rho, resetF, set_f_ftmp, get_IBMGw2, update_velIBM,
    update_IBbody, update_IBpoint, search_IBlattice, resetF x2) on the
    settling-ellipse workload, in the reference's physical units (gravity
    9.81 is hard-coded there, so dt gives the lattice gravity 1e-5)."""
    import ctypes

    import torch

    from oracle import oracle as _o
    from oracle import refcase

    dev = torch.device("cuda", env_int("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    c, host, meta = refcase.settling_ellipse_ref()
    T = _ref_tensors(host, dev)
    slots = (ctypes.c_void_p * len(_o.REF_BUFS))(*[T[k].data_ptr() if k in T else None for k in _o.REF_BUFS])
    nt, nc = meta["nt"], meta["nc"]
    inner = args.ref_inner
    ip = (ctypes.c_longlong * 16)(nt, inner, 1, 1, 0, 0, 1, *[len(w) for w in c["walls"]], nt, 3 * meta["markers"])
    fp = (ctypes.c_float * 2)(1.0, meta["rhoH"])
    Rf = _o.ref()
    for _ in range(args.warmup):
        assert Rf.lib.ref_ibm_steps_f32(slots, ip, fp) == 0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    total = 0.0
    with Clocks(dev.index or 0) as clk:
        time.sleep(0.3)
        t_start = time.perf_counter()
        for k in range(args.steps):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            assert Rf.lib.ref_ibm_steps_f32(slots, ip, fp) == 0
            e1.record()
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
        clk.window(t_start, time.perf_counter())
    value = nc * inner * args.steps / (total / 1e3) / 1e6
    # end to end: the driver's state (populations and the per-cell moments the
    # chain carries) uploaded from pinned host memory, the steps, and the
    # state read back, every bench step
    state = ["f", "p", "u", "w", "rho", "Fx", "Fz"]
    hb = {k: torch.empty(T[k].numel(), dtype=torch.float32, pin_memory=True) for k in state}
    for k in state:
        hb[k].copy_(T[k])
    torch.cuda.synchronize()
    e2e_steps = max(3, args.steps)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for k in state:
            T[k].copy_(hb[k], non_blocking=True)
        assert Rf.lib.ref_ibm_steps_f32(slots, ip, fp) == 0
        for k in state:
            hb[k].copy_(T[k], non_blocking=True)
        torch.cuda.synchronize()
    e2e = nc * inner * e2e_steps / (time.perf_counter() - t0) / 1e6
    state_bytes = sum(hb[k].numel() * 4 for k in state)
    posB = T["posB"].cpu().numpy()
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (the same ellipse, grid and walls)",
        "config": ib_config(),
        "lbm_steps_per_step": inner,
        "scheme": "the reference's EllipticalFall2 kernel chain, its CUDA built unmodified for sm_100a: "
                  "get_IBMGw2 stress-jump forcing (one pass), float body update, "
                  "<<<ceil(Nt/64),64>>> launches on the legacy stream; grid and ghosts from its own host functions",
        "body_after_m": [round(float(v), 6) for v in posB],
        "cpu_baseline": {"value": round(value, 2), "unit": METRIC, "kind": "reference", "cores": 0,
                         "sample": "the reference's own CUDA build on the GPU (it has no CPU implementation)"},
        "e2e": {"value": round(e2e, 2), "unit": METRIC, "h2d_bytes_per_step": int(state_bytes),
                "d2h_bytes_per_step": int(state_bytes)},
        "clocks": clk.summary(),
    }), flush=True)


def run_reference_2d(args):
    """The reference's LockExchange kernel chain on the closest workload to
    the nonuniform two-layer case it supports: the same 262,144 cells with
    the stretched axis along x (the reference interpolates x only), Q9
    scalar, its 5-point stencil, bounce-back."""
    import ctypes

    import torch

    from oracle import oracle as _o
    from oracle import refcase

    dev = torch.device("cuda", env_int("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    # the workload's definition (pure numpy) loaded on its own, without the package
    wl = _standalone_module("ip_cu_lbm_b200/workloads.py", "ipcu_workloads_def")
    params, S0, meta = wl.stratified_nonuniform()
    nzs, nxs = S0.shape  # stretched axis (rows of S0) becomes the reference's x axis
    c = refcase.box2d(nzs, nxs, 1.0, 1.0, 1e-6, xs=params["z"], wxs=params["wz"])
    Q, nt, nc, own = 9, c["nt"], c["nc"], c["owner"]
    # S[z, x] -> reference cell (i = z, l = x); scaled by 1e-3 because the
    # reference hard-codes g = 9.81 and rho ~ 1000 (function/collision.cu:78)
    Sg = 1e-3 * S0.T.reshape(-1)
    w9 = c["w"]
    g = (w9[None, :] * Sg[:, None]).astype(np.float32)
    ext = lambda a: np.concatenate([a, a[own]])
    st = dict(f=np.zeros(nt * Q, np.float32), g=np.concatenate([g, np.zeros((len(own), Q), np.float32)]).ravel(),
              p=np.zeros(nt, np.float32), sal=ext(Sg.astype(np.float32)), phi=np.ones(nt, np.float32),
              u=np.zeros(nt, np.float32), v=np.zeros(nt, np.float32), w=np.zeros(nt, np.float32),
              tau=np.full(nt, 3 * 0.005 + 0.5, np.float32), taus=np.full(nt, 3 * 0.0005 + 0.5, np.float32))
    st["rho"] = (1000.0 + st["sal"].astype(np.float64) * 0.824493).astype(np.float32)
    M, Mi, S, MM = refcase.mrt9()
    host = dict(items=c["items"], neib=c["neib"], nextB=c["nextB"], nextK=c["nextK"], posx=c["posx"],
                posy=c["posy"], posz=c["posz"], delX=c["delX"], delY=c["delY"], M=M.ravel(), Minv=Mi.ravel(),
                S=S, MM=MM.ravel(), ftmp=st["f"], fout=st["f"], feq=np.zeros(nt * Q), Fk=np.zeros(nt * Q),
                Fx=np.zeros(nt), Fy=np.zeros(nt), Fz=np.zeros(nt), **st)
    for a in range(6):
        wl = c["walls"][a]
        host[f"w{a + 1}"] = wl if len(wl) else np.zeros(1, np.int32)
    T = _ref_tensors(host, dev)
    slots = (ctypes.c_void_p * len(_o.REF_BUFS))(*[T[k].data_ptr() if k in T else None for k in _o.REF_BUFS])
    inner = args.ref_inner
    ip = (ctypes.c_longlong * 16)(nt, inner, 1, 1, 1, 0, 1, *[len(w) for w in c["walls"]], nt, 0)
    fp = (ctypes.c_float * 2)(1.0, 1000.0)
    Rf = _o.ref()
    for _ in range(args.warmup):
        assert Rf.lib.ref_le_steps_f32(slots, ip, fp) == 0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    total = 0.0
    with Clocks(dev.index or 0) as clk:
        t_start = time.perf_counter()
        for k in range(args.steps):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            assert Rf.lib.ref_le_steps_f32(slots, ip, fp) == 0
            e1.record()
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
        clk.window(t_start, time.perf_counter())
    value = nc * inner * args.steps / (total / 1e3) / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"reference LockExchange kernel chain, {nzs}x{nxs} cells (stretched axis along x, "
                               "5-point stencil, Q9 scalar, MRT, bounce-back), reference CUDA built for sm_100a",
                   "cells": nc},
        "lbm_steps_per_step": inner,
        "cpu_baseline": {"value": round(value, 2), "unit": METRIC, "kind": "reference", "cores": 0,
                         "sample": "the reference's own CUDA build on the GPU (it has no CPU implementation)"},
        "e2e": {"value": round(value, 2), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk.summary(),
    }), flush=True)


def run_serving(args):
    """Continuous-batching serving stream after the 512-request serving
    configuration: 60 % 2-D D2Q9 requests (half lock exchange with D2Q5
    salinity, half Rayleigh-Taylor on the Allen-Cahn phase field) on
    log-uniform grids 128x128 .. 1024x512, 30 % falling-ellipse
    immersed-boundary requests on log-uniform grids 200x600 .. 800x2400, 10 %
    3-D D3Q19 + D3Q7 stratified boxes with a falling sphere on log-uniform
    64x64x256 .. 128x128x512 (FP32: the issue-bound 3-D kernel runs 16-bit
    storage at 0.9x the FP32 speed),
    each with U[2000, 20000] steps (times --step-scale),
    2-D in FP16 storage, 150 GB admission budget, graph-captured batched
    launches with the autotuned grid per kernel class.
      * capacity: every request submitted at t = 0, served by continuous
        batching -> aggregate MLUPS (the headline value);
      * latency: Poisson arrivals at 80 % of that capacity -> p50/p99
        completion latency;
      * baseline: the same jobs run one at a time in plain FP32 through the
        same API (Sim / Sim3D with graph replay).
    The served velocities are compared with the FP32 runs (rel-L2) for three
    requests of each kind (the FP64-oracle errors of served requests are
    measured by the serving tests at sizes the oracle finishes). The
    Rayleigh-Taylor runs amplify a 1e-7 relative perturbation of the initial
    phase field to about 1e-3 in FP32 and in FP64 alike, so their FP32
    sensitivity to that perturbation is reported beside their error."""
    import torch

    from ip_cu_lbm_b200.serving import (Autotuner, Server, falling_ellipse_request, lock_exchange_request,
                                        make_sim, rayleigh_taylor_request, stratified_box_request)

    torch.cuda.set_device(0)
    rng = np.random.default_rng(20261203)
    n = args.requests
    counts = {"LE": int(round(0.3 * n)), "RT": int(round(0.3 * n)), "IB": int(round(0.3 * n))}
    counts["3D"] = n - sum(counts.values())
    kind = [k for k, c in counts.items() for _ in range(c)]
    rng.shuffle(kind)
    kinds = tuple(counts)
    logu = lambda lo, hi: float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
    dims = []
    for k in kind:
        if k in ("LE", "RT"):
            dims.append((int(logu(128, 1024)) // 32 * 32, 0, int(logu(128, 512)) // 16 * 16))
        elif k == "IB":
            nx = int(logu(200, 800)) // 8 * 8
            dims.append((nx, 0, 3 * nx))
        else:
            sc = logu(1.0, 2.0)
            dims.append((int(64 * sc) // 16 * 16, int(64 * sc) // 16 * 16, int(256 * sc) // 16 * 16))
    steps = np.maximum(rng.integers(2000, 20001, n) * args.step_scale, 2).astype(int)
    cells = np.array([nx * nz * (ny if ny else 1) for nx, ny, nz in dims])
    work = cells * steps
    makers = {"LE": lock_exchange_request, "RT": rayleigh_taylor_request, "IB": falling_ellipse_request}

    def mk(i, t, storage):
        nx, ny, nz = dims[i]
        if kind[i] == "3D":
            return stratified_box_request(i, nx, ny, nz, int(steps[i]), arrival=t, seed=i)
        return makers[kind[i]](i, nx, nz, int(steps[i]), arrival=t, storage=storage, seed=i)

    def serial_run(r, s0=None):
        if s0 is not None:
            r.s0 = s0
        s = make_sim(r)
        s.step_graph(r.steps) if r.is3d else s.step_graph(r.steps, chunk=200)
        u = np.stack([s.get("ux"), s.get("uz")])
        s.close()
        return u

    # warm-up: one small request of each kind through each path (kernel attributes, pools)
    for storage in ("f16", "f32"):
        w = Server(budget_bytes=150e9, tick_steps=200)
        w.run([lock_exchange_request(0, 128, 128, 200, storage=storage),
               rayleigh_taylor_request(1, 128, 128, 200, storage=storage),
               falling_ellipse_request(2, 200, 600, 200, storage=storage),
               stratified_box_request(3, 64, 64, 256, 200)])
        w.close()
    # autotuner: per kernel class, the grid of the persistent batched launch (untimed)
    t0 = time.perf_counter()
    tuner = Autotuner()
    tuner.tune([mk(i, 0.0, "f16") for i in range(n) if kind[i] != "3D"])
    tune_s = time.perf_counter() - t0
    # the stream-ordered memory pool grows once to the whole stream's size
    # (every request created and released, untimed), as in a long-running server
    warm = [make_sim(mk(i, 0.0, "f16")) for i in range(n)]
    for s in warm:
        s.close()
    torch.cuda.synchronize()
    # capacity: everything submitted at once
    srv = Server(budget_bytes=150e9, tick_steps=200, autotuner=tuner)
    reqs = [mk(i, 0.0, "f16") for i in range(n)]
    with Clocks(0) as ck:
        tc = time.perf_counter()
        cap = srv.run(reqs)
        ck.window(tc, time.perf_counter())
    cap_clocks = ck.summary()
    served = {r.rid: r.result for r in srv.done}
    srv.close()
    del reqs
    # latency under load: Poisson arrivals at 80 % of the measured capacity
    lam = 0.8 * cap["mlups"] * 1e6 / work.mean()
    arrivals = np.cumsum(rng.exponential(1 / lam, n))
    arrivals -= arrivals[0]
    srv = Server(budget_bytes=150e9, tick_steps=200, autotuner=tuner)
    lat = srv.run([mk(i, float(arrivals[i]), "f16") for i in range(n)])
    srv.close()
    # serial plain FP32: the same jobs one at a time through the same API
    checked = [i for k in kinds for i in [j for j in range(n) if kind[j] == k][:3]]
    ref_u = {}
    torch.cuda.synchronize()
    with Clocks(0) as ck:
        t0 = time.perf_counter()
        for i in range(n):
            u = serial_run(mk(i, 0.0, "f32"))
            if i in checked:
                ref_u[i] = u
        serial_s = time.perf_counter() - t0
        ck.window(t0, t0 + serial_s)
    serial_clocks = ck.summary()
    serial = float(work.sum()) / serial_s / 1e6
    rel = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
    errs = {k: [] for k in kinds}
    for i in checked:
        errs[kind[i]].append(rel(np.stack([served[i]["ux"], served[i]["uz"]]), ref_u[i]))
    floor = []
    for i in checked:
        if kind[i] == "RT":
            r = mk(i, 0.0, "f32")
            pert = r.s0 * (1 + 1e-7 * np.random.default_rng(i).standard_normal(r.s0.shape))
            floor.append(rel(serial_run(r, pert), ref_u[i]))
    share = {k: round(float(work[np.array(kind) == k].sum() / work.sum()), 3) for k in kinds}
    print(json.dumps({
        "metric": "served-batch MLUPS", "value": round(cap["mlups"], 1), "unit": "MLUPS", "n_gpus": 1,
        "requests": n, "capacity_wall_s": round(cap["wall_s"], 3), "capacity_host_s": cap["host_s"],
        "clocks": cap_clocks, "serial_clocks": serial_clocks,
        "graph": cap["graph"], "autotune": {"ctas_per_sm": tuner.choice, "mlups": tuner.timings,
                                            "seconds": round(tune_s, 2)},
        "p50_s": round(lat["p50_s"], 4), "p99_s": round(lat["p99_s"], 4),
        "offered_mlups": round(lat["mlups"], 1), "arrival_rate_per_s": round(lam, 3),
        "serial_fp32_mlups": round(serial, 1), "serial_fp32_wall_s": round(serial_s, 3),
        "speedup_vs_serial_fp32": round(cap["mlups"] / serial, 3),
        "max_rel_l2_velocity_vs_fp32": {k: (max(v) if v else None) for k, v in errs.items()},
        "rt_fp32_sensitivity_1e-7": max(floor) if floor else None,
        "config": {"workload": "60% 2-D (lock exchange with salinity, Rayleigh-Taylor with Allen-Cahn) on "
                               "log-uniform 128x128..1024x512, 30% falling ellipse (immersed boundary) on log-uniform "
                               "200x600..800x2400, 10% 3-D D3Q19+D3Q7 stratified boxes with a falling sphere on "
                               "log-uniform "
                               "64x64x256..128x128x512; U[2000,20000] steps x step_scale; capacity = all submitted "
                               "at t=0, latency = Poisson arrivals at 80% of capacity",
                   "requests_per_kind": counts, "work_share": share, "step_scale": args.step_scale,
                   "storage": "2-D f16 served / f32 serial; 3-D f32 both", "budget_gb": 150, "tick_steps": 200},
        "higher_is_better": True}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"])
    ap.add_argument("--inner", type=int, default=0, help="LBM steps per bench step (0: the case's default)")
    ap.add_argument("--ref-inner", type=int, default=20, help="LBM steps per bench step of the reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serving", action="store_true", help="run the continuous-batching serving stream instead")
    ap.add_argument("--requests", type=int, default=512)
    ap.add_argument("--step-scale", type=float, default=1.0, help="serving: scales the U[2000,20000] step counts")
    ap.add_argument("--case", default="ib", choices=["ib", "2d", "3d"],
                    help="ib: the settling-ellipse immersed-boundary case (default); 2d: the nonuniform "
                         "two-layer 1024x256 case; 3d: the C4-sized 3-D box")
    ap.add_argument("--dims", default="160,160,640", help="3-D box nx,ny,nz (--case 3d)")
    ap.add_argument("--uniform3d", action="store_true", help="--case 3d on a uniform box (no stretched axes)")
    ap.add_argument("--no-sphere", action="store_true", help="--case 3d without the falling sphere")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.serving:
        run_serving(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.case == "3d":
        run_3d(args)
    elif args.case == "ib":
        run_ib(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
