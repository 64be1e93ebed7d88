"""ORACLE -- test infrastructure only (bench.py's reference arm, tests).

Builds the reference driver's set-up for the settling-ellipse case (and any
2-D box) WITHOUT this repository's library: the box numbering and neighbour
table are restated in numpy (ref: EllipticalFall2/EllipticalFallxz.cu:121-170,
LockExchange/LockExchange.cu:117-127), and the ghost cells, wall lists, slip
tables, lattice constants and MRT matrices come from the reference's own
host functions compiled into oracle/_ref/libipcu_ref.so (set_neibghor_wall,
set_walln, set_bound2D, Items::setc, set_M). The moving-body arrays follow
the driver's initialisation (EllipticalFallxz.cu:188-256). Only libipcu_ref.so
is loaded, so a process that uses this module runs the reference's code and
nothing of the product's.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import sys

import numpy as np

from . import oracle as _o

# items[] slot order (ref: itemIndex.hpp:4-33)
IDX = dict(dz=0, dt=1, c=2, nx=3, ny=4, nz=5, Q=6, ratiox=7, ratioy=8, PFthick=9, num_calc=10,
           num_wall=11, num_IBPoints=12, dIBM=13, nu=14, alpha=15, sigma=16, tau=17, taus=18, wall1=19, vec=25)
EX9 = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
EZ9 = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])


@contextlib.contextmanager
def _stdout_to_stderr():
    """The reference's host set-up prints progress to stdout (Items::setc);
    send it to stderr so that a caller's stdout stays one JSON line."""
    sys.stdout.flush()
    libc = ctypes.CDLL(None)
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)


def box2d(*args, **kw):
    with _stdout_to_stderr():
        return _box2d(*args, **kw)


def _box2d(nx, nz, dx, dt, nu, n_ib=0, xs=None, wxs=None):
    """nx x nz D2Q9 box (x-z plane, ny = 1) in the driver's layout: cells
    x-major with z fastest, the neighbour table with -1 holes, then one
    ghost per boundary cell from the reference's set_neibghor_wall. x is
    uniform unless xs / wxs give the cell centres and widths along x (in
    units of dx; the reference accepts any posx/delX with delX >= dz)."""
    R = _o.ref().lib
    Q = 9
    nc = nx * nz
    I = np.repeat(np.arange(nx), nz)
    L = np.tile(np.arange(nz), nx)
    a = I[:, None] + EX9[None, :]
    d = L[:, None] + EZ9[None, :]
    inside = (a >= 0) & (a < nx) & (d >= 0) & (d < nz)
    neib0 = np.where(inside, a * nz + d, -1).astype(np.int32).ravel()
    lnum = np.arange(nc, dtype=np.int32)
    if xs is None:
        posx = ((I + 0.5) * dx).astype(np.float32)
        delX = np.full(nc, dx, np.float32)
    else:
        posx = (np.asarray(xs, np.float64)[I] * dx).astype(np.float32)
        delX = (np.asarray(wxs, np.float64)[I] * dx).astype(np.float32)
    posz = ((L + 0.5) * dx).astype(np.float32)
    posy = np.full(nc, 0.5 * dx, np.float32)
    delY = np.full(nc, dx, np.float32)
    zero = np.zeros(nc, np.float32)
    cell_in = [zero, zero, zero, posx, posy, posz, delX, delY, zero, zero, zero]
    q_in = [np.zeros(nc * Q, np.float32) for _ in range(3)]
    cap = nc + 2 * (nx + nz) + 8
    neib = np.zeros(cap * Q, np.int32)
    cell_out = [np.zeros(cap, np.float32) for _ in range(11)]
    q_out = [np.zeros(cap * Q, np.float32) for _ in range(3)]
    CP = ctypes.c_void_p
    divx = np.ones(nx, np.int32)
    divy = np.ones(1, np.int32)
    nt = R.ref_set_neibghor_wall_f32(nx, 1, nz, Q, nc, lnum.ctypes.data, divx.ctypes.data, divy.ctypes.data,
                                     neib0.ctypes.data, (CP * 11)(*[x.ctypes.data for x in cell_in]),
                                     (CP * 3)(*[x.ctypes.data for x in q_in]), cap, neib.ctypes.data,
                                     (CP * 11)(*[x.ctypes.data for x in cell_out]),
                                     (CP * 3)(*[x.ctypes.data for x in q_out]))
    if nt < 0:
        raise RuntimeError("reference set_neibghor_wall: capacity too small")
    nw = nt - nc
    neib = neib[: nt * Q].copy()
    owner = neib.reshape(-1, Q)[nc:nt, 0].copy()
    c, tau, taus = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    cx, cy, cz, w = (np.zeros(27) for _ in range(4))
    R.ref_setc(Q, dx, dt, 9, ctypes.byref(c), ctypes.byref(tau), ctypes.byref(taus), cx.ctypes.data,
               cy.ctypes.data, cz.ctypes.data, w.ctypes.data)
    items = np.zeros(25 + 4 * Q, np.float64)
    items[IDX["dz"]], items[IDX["dt"]], items[IDX["c"]] = dx, dt, c.value
    items[IDX["nx"]], items[IDX["ny"]], items[IDX["nz"]], items[IDX["Q"]] = nx, 1, nz, Q
    items[IDX["ratiox"]] = items[IDX["ratioy"]] = 1.0
    items[IDX["PFthick"]] = 3.5 * dx
    items[IDX["num_calc"]], items[IDX["num_wall"]] = nc, nw
    items[IDX["num_IBPoints"]], items[IDX["dIBM"]] = n_ib, dx
    items[IDX["nu"]], items[IDX["alpha"]] = nu, 1e-9
    items[IDX["tau"]], items[IDX["taus"]] = tau.value, taus.value
    items[25: 25 + Q], items[25 + Q: 25 + 2 * Q] = w[:Q], cx[:Q]
    items[25 + 2 * Q: 25 + 3 * Q], items[25 + 3 * Q: 25 + 4 * Q] = cy[:Q], cz[:Q]
    it = items.astype(np.float32)
    walls = [np.zeros(max(nc, 1), np.int32) for _ in range(6)]
    sizes = np.zeros(6, np.int32)
    rc = R.ref_set_walln_f32(it.ctypes.data, len(it), neib.ctypes.data, len(neib), nc,
                             (CP * 6)(*[x.ctypes.data for x in walls]), sizes.ctypes.data)
    if rc != 0:
        raise RuntimeError("reference set_walln failed")
    walls = [walls[k][: sizes[k]].copy() for k in range(6)]
    items[IDX["wall1"]: IDX["wall1"] + 6] = sizes
    it = items.astype(np.float32)
    nextK = np.zeros(max(nw, 1) * Q, np.int32)
    nextB = np.zeros(max(nw, 1) * Q, np.int32)
    R.ref_set_bound_f32(2, it.ctypes.data, len(it), nc, neib.ctypes.data, len(neib), nextK.ctypes.data,
                        nextB.ctypes.data)
    geo = {k: cell_out[i][:nt].copy() for i, k in ((3, "posx"), (4, "posy"), (5, "posz"), (6, "delX"), (7, "delY"))}
    return dict(Q=Q, nc=nc, nw=nw, nt=nt, NX=nx, NY=1, nz=nz, items=it, neib=neib, owner=owner, walls=walls,
                nextK=nextK, nextB=nextB, c=c.value, w=w[:Q], **geo)


def mrt9():
    """The reference's D2Q9 MRT matrices from its own input files via its set_M."""
    R = _o.ref().lib
    Q = 9
    M, S, Mi, MM = np.zeros((Q, Q)), np.zeros(Q), np.zeros((Q, Q)), np.zeros((Q, Q))
    if R.ref_set_M_f64(_o.REF_INPUT_DIR.encode(), Q, M.ctypes.data, S.ctypes.data, Mi.ctypes.data,
                       MM.ctypes.data) != 0:
        raise RuntimeError("reference set_M failed (oracle/_ref/input missing?)")
    return M, Mi, S, MM


def ellipse_arclength(n, a, b, samples=10000):
    """n points at equal arc length on (a cos t, b sin t) from t = 0, the
    marker layout of the reference's make_ellipce.py."""
    t = np.linspace(0.0, 2 * np.pi, samples)
    s = np.cumsum(np.hypot(-a * np.sin(t), b * np.cos(t))) * (2 * np.pi / samples)
    s -= s[0]
    tt = np.interp(np.linspace(0.0, s[-1], n, endpoint=False), s, t)
    return np.stack([a * np.cos(tt), np.zeros(n), b * np.sin(tt)], axis=1)


def quat_rot(q):
    q0, q1, q2, q3 = q
    return np.array([[q0 * q0 - q2 * q2 - q3 * q3 + q1 * q1, 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)],
                     [2 * (q1 * q2 + q0 * q3), q0 * q0 - q3 * q3 - q1 * q1 + q2 * q2, 2 * (q2 * q3 - q0 * q1)],
                     [2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3]])


def settling_ellipse_ref(nx=800, nz=3000, a_cells=20.0, b_cells=10.0, markers=240, tilt_deg=45.0, rho_ratio=1.1,
                         nu_lattice=0.02, g_lattice=1e-5, centre=(0.5, 0.85), dx=1e-3, rhoH=1000.0):
    """The settling-ellipse workload in the reference's physical units. The
    reference hard-codes gravity 9.81 m/s^2 (ref: function/ibm.cu:391), so
    dt is chosen to give the lattice gravity g dt^2/dx = g_lattice, and the
    relaxation time follows the lattice viscosity, tau = 3 nu + 1/2
    (EllipticalFallxz.cu:145). Returns (case, host buffers of the driver)."""
    dt = float(np.sqrt(g_lattice * dx / 9.81))
    nu = nu_lattice * dx * dx / dt
    c = box2d(nx, nz, dx, dt, nu, n_ib=markers)
    nt, nc, Q = c["nt"], c["nc"], 9
    a, b = a_cells * dx, b_cells * dx
    op = ellipse_arclength(markers, a, b)
    ang = np.deg2rad(tilt_deg) / 2
    q = np.array([np.cos(ang), 0.0, np.sin(ang), 0.0])
    Rm = quat_rot(q)
    posB = np.array([centre[0] * nx * dx, 0.5 * dx, centre[1] * nz * dx])
    onB = np.stack([2 * op[:, 0], np.zeros(markers), 2 * op[:, 2]], axis=1)
    onB /= np.linalg.norm(onB, axis=1)[:, None]
    posw = posB[None, :] + op @ Rm.T
    nB = onB @ Rm.T
    length = float(np.sum(np.hypot(np.diff(op[:, 0]), np.diff(op[:, 2]))))
    items = c["items"].astype(np.float64)
    items[IDX["dIBM"]] = length / markers
    c["items"] = items.astype(np.float32)
    # nearest fluid cell of each marker; the box is uniform, so it is the
    # cell whose centre is the marker's position rounded to the lattice
    I = np.clip(np.floor(posw[:, 0] / dx), 0, nx - 1).astype(np.int64)
    L = np.clip(np.floor(posw[:, 2] / dx), 0, nz - 1).astype(np.int64)
    lid = (I * nz + L).astype(np.int32)
    densB = rho_ratio * rhoH
    massB = densB * a * b * np.pi
    inertia = np.full(3, massB * (a * a + b * b) / 4)
    f32 = lambda v: np.ascontiguousarray(v, dtype=np.float32).ravel()
    tau = 3.0 * nu_lattice + 0.5
    M, Mi, S, MM = mrt9()
    host = dict(
        items=c["items"], neib=c["neib"], nextB=c["nextB"], nextK=c["nextK"], posx=c["posx"], posy=c["posy"],
        posz=c["posz"], delX=c["delX"], delY=c["delY"], M=f32(M), Minv=f32(Mi), S=f32(S), MM=f32(MM),
        f=np.zeros(nt * Q, np.float32), ftmp=np.zeros(nt * Q, np.float32), fout=np.zeros(nt * Q, np.float32),
        feq=np.zeros(nt * Q, np.float32), Fk=np.zeros(nt * Q, np.float32), g=np.zeros(nt * Q, np.float32),
        p=np.zeros(nt, np.float32), sal=np.zeros(nt, np.float32), phi=np.ones(nt, np.float32),
        tau=np.full(nt, tau, np.float32), taus=np.full(nt, 0.5, np.float32),
        Fx=np.zeros(nt, np.float32), Fy=np.zeros(nt, np.float32), Fz=np.zeros(nt, np.float32),
        rho=np.full(nt, rhoH, np.float32), u=np.zeros(nt, np.float32), v=np.zeros(nt, np.float32),
        w=np.zeros(nt, np.float32), uo=np.zeros(nt, np.float32), vo=np.zeros(nt, np.float32),
        wo=np.zeros(nt, np.float32),
        lid=lid, massB=f32([massB]), densB=f32([densB]), inertia=f32(inertia), FB=f32(np.zeros(3)),
        posB=f32(posB), Torque=f32(np.zeros(3)), velB=f32(np.zeros(3)), quat=f32(q), quaS=f32(Rm.ravel()),
        angleVB=f32(np.zeros(3)), posw=f32(posw), oposw=f32(op), Gw=f32(np.zeros(3 * markers)),
        velw=f32(np.zeros(3 * markers)), nB=f32(nB), onB=f32(onB), quatold=f32(q))
    for k in range(6):
        wl = c["walls"][k]
        host[f"w{k + 1}"] = wl if len(wl) else np.zeros(1, np.int32)
    meta = dict(dx=dx, dt=dt, nu=nu, c=c["c"], nc=nc, nt=nt, markers=markers, rhoH=rhoH)
    return c, host, meta
