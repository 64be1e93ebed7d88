"""Host-side case builders in the reference's data layout.

The reference drivers number the fluid cells of a box x-major, then y, then
z (z fastest), append one ghost ("wall lattice") cell per boundary cell, and
pack every scalar into a float items[] block (ref:
LockExchange/LockExchange.cu:34-164, function/basic.cu:203-237,
itemIndex.hpp:4-33). `box_case` reproduces that set-up through the C-ABI
host helpers of libipcu so the reference-compatible kernel entries, the
reference itself and the oracle can all run on identical inputs.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

IDX = dict(dz=0, dt=1, c=2, nx=3, ny=4, nz=5, Q=6, ratiox=7, ratioy=8, PFthick=9, num_calc=10,
           num_wall=11, num_IBPoints=12, dIBM=13, nu=14, alpha=15, sigma=16, tau=17, taus=18,
           wall1=19, vec=25)


def d2q9_mrt():
    """Lallemand-Luo D2Q9 moment basis in the reference's x-z velocity order
    (rho, e, eps, jx, qx, jz, qz, pxx, pxz), its inverse and unit rates, the
    matrices the reference reads from input/{MRT,Minv,S}_D3Q9.csv."""
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], float)
    ez = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], float)
    e2 = ex * ex + ez * ez
    M = np.stack([np.ones(9), -4 + 3 * e2, 4 - 10.5 * e2 + 4.5 * e2 * e2, ex, (-5 + 3 * e2) * ex, ez,
                  (-5 + 3 * e2) * ez, ex * ex - ez * ez, ex * ez])
    return M, np.linalg.inv(M), np.ones(9)


def setc(Q: int, dx: float, dt: float, alpha: int = 9):
    """Items::setc through the C ABI: c, tau, taus and c-scaled vectors."""
    L = _lib.lib()
    c, tau, taus = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    cx, cy, cz, w = (np.zeros(27) for _ in range(4))
    _lib.check(L.ipcu_setc(Q, dx, dt, alpha, ctypes.byref(c), ctypes.byref(tau), ctypes.byref(taus),
                           cx.ctypes.data, cy.ctypes.data, cz.ctypes.data, w.ctypes.data), "ipcu_setc")
    return c.value, tau.value, taus.value, cx[:Q], cy[:Q], cz[:Q], w[:Q]


def set_M(Q: int, M, S, Minv):
    L = _lib.lib()
    M_in, S_in, Mi_in = (np.ascontiguousarray(a, dtype=np.float64) for a in (M, S, Minv))
    Mo, So, Mio, MM = np.zeros((Q, Q)), np.zeros(Q), np.zeros((Q, Q)), np.zeros((Q, Q))
    _lib.check(L.ipcu_set_M(Q, M_in.ctypes.data, S_in.ctypes.data, Mi_in.ctypes.data, Mo.ctypes.data,
                            So.ctypes.data, Mio.ctypes.data, MM.ctypes.data), "ipcu_set_M")
    return Mo, So, Mio, MM


def box_case(Q=9, nx0=16, nz=8, ny0=1, divx=None, divy=None, dx=1.0, dt=1.0, ratiox=1.0, ratioy=1.0,
             prec="f32", pf_thick=None, sigma=0.0, nu=1e-6, n_ib=0, dIBM=None):
    """Compacted box grid with ghosts, items[], wall lists and slip tables."""
    L = _lib.lib()
    dtype = np.float32 if prec == "f32" else np.float64
    divx = np.asarray(divx if divx is not None else [1] * nx0, np.int32)
    divy = np.asarray(divy if divy is not None else [1] * ny0, np.int32)
    NX, NY = int(divx.sum()), int(divy.sum())
    ncell = NX * NY * nz
    lnum = np.zeros(ncell, np.int32)
    neib0 = np.zeros(ncell * Q, np.int32)
    geo = [np.zeros(ncell) for _ in range(5)]
    nc = L.ipcu_build_box_grid(Q, nx0, ny0, nz, dx, ratiox, ratioy, divx.ctypes.data, divy.ctypes.data,
                               lnum.ctypes.data, neib0.ctypes.data, *[g.ctypes.data for g in geo])
    if nc < 0:
        raise _lib.IpcuError(int(nc), "ipcu_build_box_grid")
    cap = 2 * nc + 8
    neib = np.full(cap * Q, -2, np.int32)
    neib[: nc * Q] = neib0
    owner = np.zeros(cap, np.int32)
    nw = L.ipcu_set_neibghor_wall(Q, NX, NY, nz, nc, lnum.ctypes.data, neib.ctypes.data, cap, owner.ctypes.data)
    if nw < 0:
        raise _lib.IpcuError(int(nw), "ipcu_set_neibghor_wall")
    nt = nc + nw
    neib = neib[: nt * Q].copy()
    owner = owner[:nw].copy()
    ext = lambda a: np.concatenate([a, a[owner]])
    posx, posy, posz, delX, delY = (ext(g) for g in geo)
    c, tau, taus, cx, cy, cz, w = setc(Q, dx, dt)
    items = np.zeros(25 + 4 * Q, np.float64)
    items[IDX["dz"]], items[IDX["dt"]], items[IDX["c"]] = dx, dt, c
    items[IDX["nx"]], items[IDX["ny"]], items[IDX["nz"]], items[IDX["Q"]] = NX, NY, nz, Q
    items[IDX["ratiox"]], items[IDX["ratioy"]] = ratiox, ratioy
    items[IDX["PFthick"]] = pf_thick if pf_thick is not None else 3.5 * dx
    items[IDX["num_calc"]], items[IDX["num_wall"]] = nc, nw
    items[IDX["num_IBPoints"]] = n_ib
    items[IDX["dIBM"]] = dIBM if dIBM is not None else dx
    items[IDX["nu"]], items[IDX["alpha"]], items[IDX["sigma"]] = nu, 1e-9, sigma
    items[IDX["tau"]], items[IDX["taus"]] = tau, taus
    items[25: 25 + Q], items[25 + Q: 25 + 2 * Q] = w, cx
    items[25 + 2 * Q: 25 + 3 * Q], items[25 + 3 * Q: 25 + 4 * Q] = cy, cz
    # wall lists (ref: set_bound.cu:23-38) and their sizes in items[19..24]
    it = items.astype(dtype)
    walls = [np.zeros(max(nc, 1), np.int32) for _ in range(6)]
    wp = (ctypes.c_void_p * 6)(*[wl.ctypes.data for wl in walls])
    sizes = np.zeros(6, np.int32)
    fn = L.ipcu_set_walln_f32 if prec == "f32" else L.ipcu_set_walln_f64
    _lib.check(fn(it.ctypes.data, neib.ctypes.data, nc, wp, sizes.ctypes.data), "ipcu_set_walln")
    walls = [walls[a][: sizes[a]].copy() for a in range(6)]
    items[IDX["wall1"]: IDX["wall1"] + 6] = sizes
    it = items.astype(dtype)
    nextK = np.zeros(max(nw, 1) * Q, np.int32)
    nextB = np.zeros(max(nw, 1) * Q, np.int32)
    if Q == 9:
        fb = L.ipcu_set_bound2D_f32 if prec == "f32" else L.ipcu_set_bound2D_f64
    else:
        fb = L.ipcu_set_bound3D_f32 if prec == "f32" else L.ipcu_set_bound3D_f64
    _lib.check(fb(it.ctypes.data, nc, neib.ctypes.data, nextK.ctypes.data, nextB.ctypes.data), "ipcu_set_bound")
    return dict(Q=Q, nc=nc, nw=nw, nt=nt, NX=NX, NY=NY, nz=nz, items=it, neib=neib, owner=owner,
                posx=posx.astype(dtype), posy=posy.astype(dtype), posz=posz.astype(dtype),
                delX=delX.astype(dtype), delY=delY.astype(dtype), walls=walls, nextK=nextK, nextB=nextB,
                lnum=lnum, c=c, tau=tau, taus=taus, w=w, cx=cx, cy=cy, cz=cz, dtype=dtype)


def box_grid_device(Q=9, nx0=16, nz=8, ny0=1, divx=None, divy=None, dx=1.0, ratiox=1.0, ratioy=1.0,
                    prec="f32", device="cuda", stream=None):
    """Box numbering, neighbour table with ghosts and cell geometry built on
    the GPU (ipcu_build_box_device_*); the same arrays as box_case's host
    path, as torch tensors on `device`."""
    import torch

    L = _lib.lib()
    tdt = torch.float32 if prec == "f32" else torch.float64
    divx = np.asarray(divx if divx is not None else [1] * nx0, np.int32)
    divy = np.asarray(divy if divy is not None else [1] * ny0, np.int32)
    NX, NY = int(divx.sum()), int(divy.sum())
    ncell = NX * NY * nz
    cap = 2 * ncell + 8
    lnum = torch.empty(ncell, dtype=torch.int32, device=device)
    neib = torch.empty(cap * Q, dtype=torch.int32, device=device)
    owner = torch.empty(cap, dtype=torch.int32, device=device)
    geo = [torch.empty(cap, dtype=tdt, device=device) for _ in range(5)]
    nc, nw = ctypes.c_int64(), ctypes.c_int64()
    fn = getattr(L, f"ipcu_build_box_device_{prec}")
    _lib.check(fn(Q, len(divx), len(divy), nz, dx, ratiox, ratioy, divx.ctypes.data, divy.ctypes.data,
                  lnum.data_ptr(), neib.data_ptr(), *[g.data_ptr() for g in geo], cap, owner.data_ptr(),
                  ctypes.byref(nc), ctypes.byref(nw), stream), "ipcu_build_box_device")
    nt = nc.value + nw.value
    posx, posy, posz, delX, delY = (g[:nt] for g in geo)
    return dict(Q=Q, nc=nc.value, nw=nw.value, nt=nt, NX=NX, NY=NY, nz=nz, lnum=lnum, neib=neib[: nt * Q],
                owner=owner[: nw.value], posx=posx, posy=posy, posz=posz, delX=delX, delY=delY)


def nearest_cells(posx, posy, posz, num_calc, posw, stream=None):
    """lattice_id of each marker (posw: [n, 3] device tensor) on the GPU."""
    import torch

    prec = "f32" if posx.dtype == torch.float32 else "f64"
    posw = posw.contiguous()
    n = posw.numel() // 3
    lid = torch.empty(n, dtype=torch.int32, device=posw.device)
    _lib.check(getattr(_lib.lib(), f"ipcu_nearest_cells_{prec}")(
        posx.data_ptr(), posy.data_ptr(), posz.data_ptr(), int(num_calc), posw.data_ptr(), n, lid.data_ptr(),
        stream), "ipcu_nearest_cells")
    return lid


def compact_to_grid(case, a):
    """Fluid values of a 2-D (ny=1) case in compact x-major/z-fastest order ->
    [nz, nx] array (x fastest), the structured solver's layout."""
    NX, nz = case["NX"], case["nz"]
    return np.asarray(a)[: NX * nz].reshape(NX, nz).T.copy()


def grid_to_compact(case, g):
    return np.asarray(g).T.reshape(-1).copy()


def ellipse_points(n, a=1.0, b=0.5, samples=10000):
    """n points at equal arc length on the ellipse (a cos t, b sin t),
    starting at t = 0 (the marker layout of the reference's ellipse case,
    EllipticalFall2/make_ellipce.py): the arc length is accumulated on a fine
    parameter grid and inverted by linear interpolation."""
    t = np.linspace(0.0, 2 * np.pi, samples)
    ds = np.hypot(-a * np.sin(t), b * np.cos(t))
    s = np.cumsum(ds) * (2 * np.pi / samples)
    s -= s[0]
    target = np.linspace(0.0, s[-1], n, endpoint=False)
    tt = np.interp(target, s, t)
    return np.stack([a * np.cos(tt), np.zeros(n), b * np.sin(tt)], axis=1)


def quat_rot(q):
    q0, q1, q2, q3 = q
    return np.array([[q0 * q0 - q2 * q2 - q3 * q3 + q1 * q1, 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)],
                     [2 * (q1 * q2 + q0 * q3), q0 * q0 - q3 * q3 - q1 * q1 + q2 * q2, 2 * (q2 * q3 - q0 * q1)],
                     [2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3]])


def ibm_ellipse_case(nx0=40, nz=60, n_markers=24, dx=1e-3, dt=1e-3, tilt_deg=45.0, rho_ratio=1.1, rhoH=1000.0,
                     nu=1e-6, center=(0.5, 0.5), prec="f32", a_frac=1 / 8):
    """Settling-ellipse case in the reference driver's set-up
    (ref: EllipticalFall2/EllipticalFallxz.cu:45-46,188-256): semi-axes
    a = H/8, b = a/2 with H = nx*dx, markers at equal arc length, body
    rotated about y by the tilt, radial marker normals (2x, 0, 2z)/|.|,
    mass and inertia of the 2-D ellipse, each marker's lattice cell the
    nearest fluid cell. Returns (case, body) with host arrays."""
    c = box_case(Q=9, nx0=nx0, nz=nz, dx=dx, dt=dt, prec=prec, n_ib=n_markers, nu=nu)
    dtp = c["dtype"]
    H = dx * nx0
    a = H * a_frac
    b = a / 2
    op = ellipse_points(n_markers, 1.0, 0.5) * a
    ang = np.deg2rad(tilt_deg) / 2
    q = np.array([np.cos(ang), 0.0, np.sin(ang), 0.0])
    R = quat_rot(q)
    posB = np.array([center[0] * nx0 * dx, dx * 1 / 2.0, center[1] * nz * dx])
    onB = np.stack([2 * op[:, 0], np.zeros(n_markers), 2 * op[:, 2]], axis=1)
    onB /= np.linalg.norm(onB, axis=1)[:, None]
    posw = posB[None, :] + op @ R.T
    nB = onB @ R.T
    length = np.sum(np.hypot(np.diff(op[:, 0]), np.diff(op[:, 2])))
    nc = c["nc"]
    P = np.stack([c["posx"][:nc], c["posy"][:nc], c["posz"][:nc]], axis=1).astype(np.float64)
    lid = np.array([int(np.argmin(np.linalg.norm(P - pw[None, :], axis=1))) for pw in posw], np.int32)
    densB = rho_ratio * rhoH
    massB = densB * a * b * np.pi
    inertia = np.full(3, massB * (a * a + b * b) / 4)
    items = c["items"].astype(np.float64)
    items[IDX["num_IBPoints"]] = n_markers
    items[IDX["dIBM"]] = length / n_markers
    c["items"] = items.astype(dtp)
    c["n_ib"] = n_markers
    f32 = lambda v: np.ascontiguousarray(v, dtype=dtp).ravel()
    body = dict(lid=lid, massB=f32([massB]), densB=f32([densB]), inertia=f32(inertia), FB=f32(np.zeros(3)),
                posB=f32(posB), Torque=f32(np.zeros(3)), velB=f32(np.zeros(3)), quat=f32(q), quaS=f32(R.ravel()),
                angleVB=f32(np.zeros(3)), posw=f32(posw), oposw=f32(op), Gw=f32(np.zeros(3 * n_markers)),
                velw=f32(np.zeros(3 * n_markers)), nB=f32(nB), onB=f32(onB), quatold=f32(q))
    return c, body


def ellipse_markers(a, b, n):
    """Lagrangian markers of an ellipse (x/a)^2 + (z/b)^2 = 1 in the body
    frame: n points at equal arc length (dense polyline of the perimeter,
    inverted by interpolation) and the arc length each one carries."""
    t = np.linspace(0.0, 2.0 * np.pi, 40001)
    x, z = a * np.cos(t), b * np.sin(t)
    s = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(x), np.diff(z)))])
    tt = np.interp(np.arange(n) * s[-1] / n, s, t)
    return np.stack([a * np.cos(tt), b * np.sin(tt)], 1), np.full(n, s[-1] / n)


def sphere_markers(radius, n):
    """Lagrangian markers of a sphere of the given radius in the body frame:
    n points on a Fibonacci lattice (z = 1 - (2i + 1)/n, azimuth advancing by
    the golden angle), each carrying the area 4 pi R^2 / n."""
    i = np.arange(n)
    z = 1.0 - (2.0 * i + 1.0) / n
    rxy = np.sqrt(np.maximum(1.0 - z * z, 0.0))
    phi = i * (np.pi * (3.0 - np.sqrt(5.0)))
    r = radius * np.stack([rxy * np.cos(phi), rxy * np.sin(phi), z], 1)
    return r, np.full(n, 4.0 * np.pi * radius * radius / n)
