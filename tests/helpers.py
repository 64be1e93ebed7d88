"""Shared test helpers: reference-style states on compacted box grids and
step-chain runners for the oracle (CPU), the reference build (GPU, via
oracle/_ref) and the product (GPU, libipcu.so)."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from ip_cu_lbm_b200 import cases
from ip_cu_lbm_b200.lockexchange import ibm_step, le_step, pf_step

RHO_SAL = 0.824493


def rel_l2(a, b, floor=0.0):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    d = np.linalg.norm(a - b)
    n = max(np.linalg.norm(b), floor)
    return d / n if n > 0 else d


def seq_sum(a, axis_len, dtype):
    """Sum over the population index in order 0..Q-1 at precision dtype."""
    acc = np.zeros(a.shape[0], dtype)
    for k in range(axis_len):
        acc = (acc + a[:, k].astype(dtype)).astype(dtype)
    return acc


def density(S, phi, rhoL, rhoH, dtype):
    base = dtype(rhoL) + (dtype(rhoH) - dtype(rhoL)) * phi.astype(dtype)
    return (base.astype(np.float64) + S.astype(dtype).astype(np.float64) * RHO_SAL).astype(dtype)


def random_state(case, seed, *, rhoL=1.0, rhoH=1000.0, tau=0.6, taus=0.55, amp=1e-3, smin=0.0, smax=1.0,
                 noise=0.2):
    """A smooth-ish random state in the reference driver's layout: fluid
    values first, then ghosts carrying their owner's p, rho, phi (f, g, u
    zero), as set_neibghor_wall leaves them (ref: function/basic.cu:215-226)."""
    rng = np.random.default_rng(seed)
    Q, nc, nt = case["Q"], case["nc"], case["nt"]
    dt = case["dtype"]
    own = case["owner"]
    cx, cy, cz, w, c = case["cx"], case["cy"], case["cz"], case["w"], case["c"]
    # smooth fields: low-order modes of the cell position
    X, Y, Z = (case[k][:nc].astype(np.float64) for k in ("posx", "posy", "posz"))
    Lx, Lz = max(X.max(), 1e-12), max(Z.max(), 1e-12)
    ph = rng.uniform(0, 2 * np.pi, 6)
    S = smin + (smax - smin) * (0.5 + 0.5 * np.sin(2 * np.pi * X / Lx + ph[0]) * np.cos(np.pi * Z / Lz + ph[1]))
    u = amp * np.sin(2 * np.pi * Z / Lz + ph[2]) * (1 + 0.3 * rng.standard_normal(nc))
    wv = amp * np.cos(2 * np.pi * X / Lx + ph[3]) * (1 + 0.3 * rng.standard_normal(nc))
    v = amp * np.sin(ph[4] + X / Lx) * (1 if Q == 27 else 0) * np.ones(nc)
    p0 = amp * rng.standard_normal(nc)
    eu = (np.outer(u, cx) + np.outer(v, cy) + np.outer(wv, cz)) / c ** 2
    us = ((u ** 2 + v ** 2 + wv ** 2) / c ** 2)[:, None]
    f = w[None, :] * (p0[:, None] + 3 * eu + 4.5 * eu ** 2 - 1.5 * us)
    f += noise * amp * w[None, :] * rng.standard_normal((nc, Q))
    g = w[None, :] * S[:, None] * (1 + 3 * eu + 4.5 * eu ** 2 - 1.5 * us)
    g += noise * 1e-2 * w[None, :] * rng.standard_normal((nc, Q))
    f, g = f.astype(dt), g.astype(dt)
    S, u, v, wv = S.astype(dt), u.astype(dt), v.astype(dt), wv.astype(dt)
    p = seq_sum(f, Q, dt)
    phi = np.ones(nc, dt)
    rho = density(S, phi, rhoL, rhoH, dt)

    def ext(a, zero=False):
        return np.concatenate([a, np.zeros(len(own), a.dtype) if zero else a[own]])

    st = dict(
        f=np.concatenate([f, np.zeros((len(own), Q), dt)]).ravel(),
        g=np.concatenate([g, np.zeros((len(own), Q), dt)]).ravel(),
        p=ext(p), sal=ext(S), phi=ext(phi), rho=ext(rho), u=ext(u, True), v=ext(v, True), w=ext(wv, True),
        tau=np.full(nt, tau, dt), taus=np.full(nt, taus, dt),
    )
    return st


def random_pf_state(case, seed, *, rhoL=1.0, rhoH=3.0, tau=0.6, taus=0.58, amp=1e-3, noise=0.2):
    """A two-phase state: the smooth random scalar becomes the order
    parameter phi in [0.02, 0.98] (no salinity), rho the mixture density, and
    the previous-step fields phi_old, u_old equal the current ones (so the
    d(phi u)/dt term starts at zero, as in the reference driver)."""
    st = random_state(case, seed, rhoL=rhoL, rhoH=rhoH, tau=tau, taus=taus, amp=amp, smin=0.02, smax=0.98,
                      noise=noise)
    dt = case["dtype"]
    phi = st["sal"].copy()
    st["phi"] = phi
    st["sal"] = np.zeros_like(phi)
    st["rho"] = density(st["sal"], phi, rhoL, rhoH, dt)
    st["phiold"], st["uold"], st["vold"], st["wold"] = phi.copy(), st["u"].copy(), st["v"].copy(), st["w"].copy()
    return st


def mrt_mats(Q=9):
    M, Minv, S = cases.d2q9_mrt()
    _, So, _, MM = cases.set_M(Q, M, S, Minv)
    return M, Minv, So, MM


def _buffers(case, state, xp, mats=None):
    """SimpleNamespace of the driver's buffers; xp converts a numpy array."""
    Q, nt, dt = case["Q"], case["nt"], case["dtype"]
    B = SimpleNamespace()
    B.items, B.neib = xp(case["items"]), xp(case["neib"])
    B.nextB, B.nextK = xp(case["nextB"]), xp(case["nextK"])
    for k in ("posx", "posy", "posz", "delX", "delY"):
        setattr(B, k, xp(case[k]))
    for k in ("f", "g", "p", "sal", "phi", "rho", "tau", "taus", "u", "v", "w"):
        setattr(B, k, xp(state[k]))
    B.ftmp, B.fout = xp(state["f"]), xp(state["f"])
    B.feq, B.Fk = xp(np.zeros(nt * Q, dt)), xp(np.zeros(nt * Q, dt))
    B.Fx, B.Fy, B.Fz = (xp(np.zeros(nt, dt)) for _ in range(3))
    if mats is not None:
        B.M, B.Minv, B.S, B.MM = (xp(np.ascontiguousarray(m, dtype=dt).ravel()) for m in mats)
    else:
        B.M = B.Minv = B.S = B.MM = None
    for a, wl in enumerate(case["walls"]):
        setattr(B, f"w{a + 1}", xp(wl if len(wl) else np.zeros(1, np.int32)))
    for k, v in state.items():
        if not hasattr(B, k):
            setattr(B, k, xp(v))
    return B


def oracle_chain(case, state, nsteps, *, prec=None, slip=1, mats=None, kind="le", **kw):
    """Runs the driver order on the CPU oracle; returns the buffer namespace (numpy)."""
    from oracle import oracle as _o

    O = _o.oracle()
    prec = prec or ("f32" if case["dtype"] == np.float32 else "f64")
    dt = np.float32 if prec == "f32" else np.float64
    xp = lambda a: np.ascontiguousarray(a, dtype=dt if np.asarray(a).dtype.kind == "f" else np.int32).copy()
    B = _buffers(case, state, xp, mats)

    def call(name, *args):
        O(name, prec, *args)

    def ip(f, feq, ftmp, fout):
        O.IP_process(prec, B.items, B.neib, f, feq, ftmp, fout, B.nextB, B.nextK, B.posx, B.posy, B.delX, B.delY,
                     slip)

    B.copy_f_ftmp = lambda: np.copyto(B.ftmp[: case["nc"] * case["Q"]], B.f[: case["nc"] * case["Q"]])
    for _ in range(nsteps):
        if kind == "le":
            le_step(call, ip, B, num_F=case["nt"], wall_sizes=tuple(len(w) for w in case["walls"]),
                    mrt=mats is not None, **kw)
        elif kind == "pf":
            pf_step(call, ip, B, num_F=case["nt"], mrt=mats is not None, **kw)
        else:
            ibm_step(call, ip, B, num_F=case["nt"], num_Gw=case["n_ib"] * 3, mrt=mats is not None, **kw)
    return B


def gpu_chain(case, state, nsteps, backend, *, slip=1, mats=None, kind="le", **kw):
    """Runs the driver order on the GPU through `backend` ("ref" = the
    reference build, "ipcu" = this library). Returns buffers as numpy."""
    import torch

    from ip_cu_lbm_b200 import _lib

    prec = "f32" if case["dtype"] == np.float32 else "f64"
    dev = torch.device("cuda:0")
    tdt = torch.float32 if prec == "f32" else torch.float64

    def xp(a):
        a = np.asarray(a)
        return torch.as_tensor(np.ascontiguousarray(a), dtype=tdt if a.dtype.kind == "f" else torch.int32,
                               device=dev).clone()

    B = _buffers(case, state, xp, mats)
    nt = case["nt"]
    if backend == "ref":
        from oracle import oracle as _o

        R = _o.ref()

        def call(name, *args):
            rc = R(name, prec, *args, n=nt)
            assert rc == 0, f"reference {name} failed: {rc}"

        def ip(f, feq, ftmp, fout):
            rc = R.IP_process(prec, B.items, B.neib, f, feq, ftmp, fout, B.nextB, B.nextK, B.posx, B.posy, B.delX,
                              B.delY, slip, nt)
            assert rc == 0

    else:
        L = _lib.legacy()
        stream = torch.cuda.current_stream(dev).cuda_stream

        def call(name, *args):
            _lib.check(L(name, prec, *args, tail=(nt, stream)), name)

        def ip(f, feq, ftmp, fout):
            fn = getattr(_lib.lib(), f"ipcu_IP_process_{prec}")
            _lib.check(fn(*[x.data_ptr() if hasattr(x, "data_ptr") else x for x in
                            (B.items, (nt + 63) // 64, 64, B.neib, f, feq, ftmp, fout, B.nextB, B.nextK, B.posx,
                             B.posy, B.delX, B.delY)], int(slip), stream), "IP_process")

    n_fl = case["nc"] * case["Q"]
    B.copy_f_ftmp = lambda: B.ftmp[:n_fl].copy_(B.f[:n_fl])
    for _ in range(nsteps):
        if kind == "le":
            le_step(call, ip, B, num_F=nt, wall_sizes=tuple(len(w) for w in case["walls"]), mrt=mats is not None,
                    **kw)
        elif kind == "pf":
            pf_step(call, ip, B, num_F=nt, mrt=mats is not None, **kw)
        else:
            ibm_step(call, ip, B, num_F=nt, num_Gw=case["n_ib"] * 3, mrt=mats is not None, **kw)
    torch.cuda.synchronize()
    out = SimpleNamespace()
    for k, v in vars(B).items():
        if hasattr(v, "detach"):
            setattr(out, k, v.detach().cpu().numpy())
    return out
