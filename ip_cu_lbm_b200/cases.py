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


def compact_to_grid(case, a):
    """Fluid values of a 2-D (ny=1) case in compact x-major/z-fastest order ->
    [nz, nx] array (x fastest), the structured solver's layout."""
    NX, nz = case["NX"], case["nz"]
    return np.asarray(a)[: NX * nz].reshape(NX, nz).T.copy()


def grid_to_compact(case, g):
    return np.asarray(g).T.reshape(-1).copy()
