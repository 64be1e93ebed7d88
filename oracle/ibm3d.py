"""ORACLE -- test infrastructure only. FP64 numpy restatement of the 3-D
moving immersed boundary on the structured 3-D oracle (oracle/structured3d.py):
a rigid sphere carrying markers on a Fibonacci lattice, multi-direct forcing
(MDF) with the reference's 4-point Peskin kernel (ref: function/ibm.cu:61-66
weightFunction) applied per axis, and the rigid-body update of the 2-D
oracle (oracle/ibm2d.py) in three dimensions: the reaction of the mean of
this and the previous step's IB force, buoyancy (1 - rho_f/rho_s) m g along
-z (ref: function/ibm.cu:383-396, update_IBbody), the change of the fluid
momentum inside the body (Kempe & Froehlich 2012) with volume fractions
clamp(1/2 - d/dz, 0, 1), d = |x - X| - R, forward Euler, the markers
following the body (ref: update_IBpoint, ibm.cu:426-447) by a rotation
matrix advanced with the mean angular velocity.

Stretched x and y axes: the Peskin kernel is evaluated in index space. A
marker at x lies at the continuous index s = i + (x - x_i)/(x_{i+1} - x_i)
between the cell centres x_i <= x < x_{i+1}; its stencil is the four cells
floor(s) - 1 .. floor(s) + 2 with weights phi(j - s) (a partition of unity
on any grid), and the force spreads as dF dA phi phi phi / V_j with V_j the
cell's volume, so the spread force sums to the marker force. On a uniform
grid this is the usual kernel.

One coupled step:
  1. fluid step with the previous IB force density f_ib in the force; the
     state's velocity u = c j + F dt/2rho carries it;
  2. MDF from u* = u - f_ib dt/2rho, `iters` times: U*_l = sum phi u*,
     dF_l = 2 rho_f (U_b,l - U*_l)/dt, df = spread, u* += df dt/2rho,
     f_ib' += df; the state's force becomes F - f_ib + f_ib', so that the
     next step's velocity is the corrected one;
  3. body update.
"""
from __future__ import annotations

import numpy as np

from oracle.ibm2d import peskin4
from oracle.structured3d import E19, Box3D


def sphere_markers(radius, n):
    """n markers on a Fibonacci lattice over the sphere |r| = radius (body
    frame) and the area each carries."""
    i = np.arange(n)
    z = 1.0 - (2.0 * i + 1.0) / n
    rxy = np.sqrt(np.maximum(1.0 - z * z, 0.0))
    phi = i * (np.pi * (3.0 - np.sqrt(5.0)))
    r = radius * np.stack([rxy * np.cos(phi), rxy * np.sin(phi), z], 1)
    return r, np.full(n, 4.0 * np.pi * radius * radius / n)


def rotation(w):
    """Rotation matrix of the rotation vector w (Rodrigues)."""
    th = float(np.linalg.norm(w))
    if th == 0.0:
        return np.eye(3)
    k = w / th
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + np.sin(th) * K + (1.0 - np.cos(th)) * (K @ K)


class Sphere3D:
    def __init__(self, xc, yc, zc, radius, n_markers, *, rho_s):
        self.X = np.array([xc, yc, zc], float)
        self.U = np.zeros(3)
        self.om = np.zeros(3)
        self.R = np.eye(3)
        self.radius = float(radius)
        self.r0, self.dA = sphere_markers(radius, n_markers)
        vol = 4.0 / 3.0 * np.pi * radius ** 3
        self.m = rho_s * vol
        self.I = 0.4 * self.m * radius * radius
        self.rho_s = rho_s
        self.P_in = self.L_in = None
        self.Fib, self.Tib = np.zeros(3), np.zeros(3)

    def markers(self):
        r = self.r0 @ self.R.T
        return self.X[None] + r, self.U[None] + np.cross(self.om[None], r), r


def index_coord(centres, x):
    """Continuous cell index of positions x on an axis with the given
    cell centres (linear between centres, clamped outside)."""
    n = len(centres)
    i = np.clip(np.searchsorted(centres, x, side="right") - 1, 0, n - 2)
    return i + (x - centres[i]) / (centres[i + 1] - centres[i])


class IBBox3D:
    def __init__(self, box: Box3D, body: Sphere3D, *, rho_f, gravity, iters=3):
        self.b, self.body = box, body
        self.rho_f, self.g, self.iters = rho_f, gravity, iters
        b = box
        self.zc = (np.arange(b.nz) + 0.5) * b.dz

    def _stencil(self, X):
        b = self.b
        sx, sy, sz = index_coord(b.X, X[:, 0]), index_coord(b.Y, X[:, 1]), index_coord(self.zc, X[:, 2])
        i0, j0, k0 = (np.floor(s).astype(int) - 1 for s in (sx, sy, sz))
        a = np.arange(64)
        I, J, K = i0[:, None] + (a & 3)[None], j0[:, None] + ((a >> 2) & 3)[None], k0[:, None] + (a >> 4)[None]
        W = peskin4(I - sx[:, None]) * peskin4(J - sy[:, None]) * peskin4(K - sz[:, None])
        ok = (I >= 0) & (I < b.nx) & (J >= 0) & (J < b.ny) & (K >= 0) & (K < b.nz)
        return (np.clip(K, 0, b.nz - 1), np.clip(J, 0, b.ny - 1), np.clip(I, 0, b.nx - 1)), np.where(ok, W, 0.0)

    def step(self, n=1):
        for _ in range(n):
            self._step()

    def _step(self):
        b, body = self.b, self.body
        b.step(1)
        p, S, rho, u = b.moments()
        h = b.dt / (2 * rho)
        us = [u[a] - b.fext[a] * h for a in range(3)]
        X, Ub, r = body.markers()
        idx, W = self._stencil(X)
        vol = (b.DX[None, None, :] * b.DY[None, :, None]) * b.dz
        Ft = np.zeros((len(X), 3))
        fib = np.zeros_like(b.fext)
        for _ in range(self.iters):
            Us = np.stack([(W * us[a][idx]).sum(1) for a in range(3)], 1)
            dF = 2 * self.rho_f * (Ub - Us) / b.dt
            wd = W * body.dA[:, None]
            for a in range(3):
                df = np.zeros(b.fext.shape[1:])
                np.add.at(df, idx, dF[:, a:a + 1] * wd)
                df = df / vol
                us[a] = us[a] + df * h
                fib[a] += df
            Ft += dF
        b.F = b.F - b.fext + fib
        b.fext = fib
        # body: reaction of the marker forces, buoyancy, fluid momentum inside
        FdA = Ft * body.dA[:, None]
        Fib = FdA.sum(0)
        Tib = np.cross(r, FdA).sum(0)
        Fb = -(Fib + body.Fib) / 2
        Tb = -(Tib + body.Tib) / 2
        body.Fib, body.Tib = Fib, Tib
        Fb[2] += -(1.0 - self.rho_f / body.rho_s) * body.m * self.g
        p, S, rho, u = b.moments()
        ZZ, YY, XX = np.meshgrid(self.zc, b.Y, b.X, indexing="ij")
        d = np.sqrt((XX - body.X[0]) ** 2 + (YY - body.X[1]) ** 2 + (ZZ - body.X[2]) ** 2) - body.radius
        al = np.clip(0.5 - d / b.dz, 0.0, 1.0) * vol
        P = np.array([(al * u[a]).sum() for a in range(3)])
        rr = [XX - body.X[0], YY - body.X[1], ZZ - body.X[2]]
        L = np.array([(al * (rr[1] * u[2] - rr[2] * u[1])).sum(), (al * (rr[2] * u[0] - rr[0] * u[2])).sum(),
                      (al * (rr[0] * u[1] - rr[1] * u[0])).sum()])
        if body.P_in is None:
            body.P_in, body.L_in = P, L
        dt = b.dt
        Uold, omold = body.U.copy(), body.om.copy()
        body.U = body.U + (dt * Fb + self.rho_f * (P - body.P_in)) / body.m
        body.om = body.om + (dt * Tb + self.rho_f * (L - body.L_in)) / body.I
        body.X = body.X + dt * (body.U + Uold) / 2
        body.R = rotation(dt * (body.om + omold) / 2) @ body.R
        body.P_in, body.L_in = P, L
