"""ORACLE -- test infrastructure only. FP64 numpy restatement of the fused
2-D path with a moving immersed boundary: one rigid body in the x-z plane,
Lagrangian markers on its outline, multi-direct forcing (MDF) with the
4-point Peskin kernel of the reference's weightFunction
(ref: function/ibm.cu:61-66), and a rigid-body update in FP64 built on the
reference's update_IBbody (ref: function/ibm.cu:367-424: force and torque
summed over the markers, buoyancy (1 - rho_f/rho_s) m g) and update_IBpoint
(ibm.cu:426-447), restricted to the plane (one rotation angle instead of a
quaternion). The reference's AB2 rule is replaced by a momentum balance
that stays stable at density ratios near one:
  * with the forcing of the fluid step, the velocity after a step carries
    half of this step's IB force and half of the previous one's, so the
    fluid's momentum changes by the MEAN of the two; the body takes the
    reaction of that mean (the reaction of this step's force alone couples
    to the force's neutral even-odd mode and grows);
  * with direct forcing the marker reaction also carries the force that
    accelerates the fluid inside the body, so the change of the fluid
    momentum inside the body is added back (Kempe & Froehlich 2012), each
    cell weighted by its volume fraction alpha = clamp(1/2 - d/dz, 0, 1),
    d the signed distance of its centre from the outline (first-order
    estimate F/|grad F| of the ellipse function F): a binary inside test
    gives the body a kick whenever a cell centre crosses the outline;
  m (U' - U) = dt (F_h + F_g) + rho_f (P_in - P_in,old),
  I (w' - w) = dt T_h + rho_f (L_in - L_in,old),
  F_h = -(F_ib + F_ib,old)/2, T_h likewise,
  X' = X + dt (U + U')/2, theta' = theta + dt (w + w')/2.

One coupled step:
  1. fluid step (structured oracle) with the previous IB force density f_ib
     added to the body force; the half of it in the new velocity is taken
     out again, so that MDF finds the whole force of this step;
  2. MDF, `iters` times: interpolate u at the markers
     (U*_l = sum_x u(x) phi(rx) phi(rz)), dF_l = 2 rho_f (U_b,l - U*_l) / dt,
     spread df(x) = sum_l dF_l phi phi dS_l / dz^2, correct
     u(x) += df dt / (2 rho(x)), accumulate f_ib += df and F_l += dF_l;
  3. body: F_b = -sum_l F_l dS_l + buoyancy, T_b = -sum_l r_l x F_l dS_l,
     momentum change of the fluid inside; markers follow the body.
The reference's own IB coupling (get_IBMGw2, a sigma-jump population
interpolation) is a different method and stays available through the
kernel-entry API; this mode has no reference counterpart beyond the shared
kernel (weightFunction) and body update rules.
"""
from __future__ import annotations

import numpy as np

from oracle.structured import Box


def peskin4(r):
    """4-point Peskin kernel phi(r), r in lattice spacings (ref: ibm.cu:61-66)."""
    r = np.abs(np.asarray(r, float))
    a = (3 - 2 * r + np.sqrt(np.clip(1 + 4 * r - 4 * r * r, 0, None))) / 8
    b = (5 - 2 * r - np.sqrt(np.clip(-7 + 12 * r - 4 * r * r, 0, None))) / 8
    return np.where(r < 1, a, np.where(r <= 2, b, 0.0))


def ellipse_markers(a, b, n):
    """n markers at equal arc length on the ellipse (x/a)^2 + (z/b)^2 = 1 (body
    frame), and the arc length each carries."""
    t = np.linspace(0, 2 * np.pi, 20001)
    x, z = a * np.cos(t), b * np.sin(t)
    s = np.concatenate([[0], np.cumsum(np.hypot(np.diff(x), np.diff(z)))])
    per = s[-1]
    tt = np.interp(np.arange(n) * per / n, s, t)
    return np.stack([a * np.cos(tt), b * np.sin(tt)], 1), np.full(n, per / n)


class Body2D:
    def __init__(self, xc, zc, X0, dS, *, rho_s, area, inertia_per_mass, theta=0.0):
        self.X = np.array([xc, zc], float)
        self.U = np.zeros(2)
        self.th, self.om = float(theta), 0.0
        self.X0, self.dS = np.asarray(X0, float), np.asarray(dS, float)
        self.m = rho_s * area
        self.I = self.m * inertia_per_mass
        self.rho_s = rho_s
        self.a_b = None  # semi-axes for the inside test (set by ellipse bodies)
        self.P_in, self.L_in = None, None  # fluid momentum / angular momentum inside, previous step
        self.Fib, self.Tib = np.zeros(2), 0.0  # IB force / torque on the fluid, previous step

    def fraction(self, xc, zc, h):
        """Volume fraction of cells (centres xc, zc, size h) inside the
        ellipse: clamp(1/2 - d/h, 0, 1), d = F/|grad F| with
        F = (x/a)^2 + (z/b)^2 - 1 in the body frame."""
        a, bb = self.a_b
        c, s = np.cos(self.th), np.sin(self.th)
        dx, dz = xc - self.X[0], zc - self.X[1]
        xb, zb = c * dx + s * dz, -s * dx + c * dz
        F = (xb / a) ** 2 + (zb / bb) ** 2 - 1.0
        G = 2.0 * np.hypot(xb / (a * a), zb / (bb * bb))
        d = F / np.maximum(G, 1e-300)
        return np.clip(0.5 - d / h, 0.0, 1.0)

    def markers(self):
        c, s = np.cos(self.th), np.sin(self.th)
        R = np.array([[c, -s], [s, c]])
        r = self.X0 @ R.T
        X = self.X[None] + r
        U = self.U[None] + self.om * np.stack([-r[:, 1], r[:, 0]], 1)
        return X, U


class IBBox:
    """The coupled step for one body or a list of bodies (each with its own
    markers, stencils and rigid-body state; they share the fluid's force
    density and must stay apart, as the GPU path requires)."""

    def __init__(self, box: Box, body, *, rho_f, gravity, iters=3):
        self.bodies = list(body) if isinstance(body, (list, tuple)) else [body]
        self.b, self.body = box, self.bodies[0]
        self.rho_f, self.g, self.iters = rho_f, gravity, iters

    def _stencil(self, X):
        """Cells (k, i) and weights of the 4x4 stencil of every marker; cells
        outside the box carry weight 0."""
        b = self.b
        xs, zs = X[:, 0] / b.dz - 0.5, X[:, 1] / b.dz - 0.5
        i0, k0 = np.floor(xs).astype(int) - 1, np.floor(zs).astype(int) - 1
        a = np.arange(16) & 3
        c = np.arange(16) >> 2
        I = i0[:, None] + a[None]
        K = k0[:, None] + c[None]
        W = peskin4(I - xs[:, None]) * peskin4(K - zs[:, None])
        ok = (I >= 0) & (I < b.nx) & (K >= 0) & (K < b.nz)
        return np.clip(K, 0, b.nz - 1), np.clip(I, 0, b.nx - 1), np.where(ok, W, 0.0)

    def step(self, n=1):
        for _ in range(n):
            self._step()

    def _step(self):
        b = self.b
        b.step(1)
        rho = b.rho_of(b.S)
        # the fluid step's velocity carries half of the previous IB force;
        # MDF starts from the velocity without it and finds the whole force
        b.ux = b.ux - b.fext[0] * b.dt / (2 * rho)
        b.uz = b.uz - b.fext[1] * b.dt / (2 * rho)
        fib = np.zeros_like(b.fext)
        for body in self.bodies:
            self._couple(body, rho, fib)
        b.fext = fib

    def _couple(self, body, rho, fib):
        b = self.b
        X, Ub = body.markers()
        K, I, W = self._stencil(X)
        Ft = np.zeros((len(X), 2))
        h2 = b.dz * b.dz
        for _ in range(self.iters):
            Us = np.stack([(W * b.ux[K, I]).sum(1), (W * b.uz[K, I]).sum(1)], 1)
            dF = 2 * self.rho_f * (Ub - Us) / b.dt
            df = np.zeros_like(fib)
            wd = W * (body.dS / h2)[:, None]
            np.add.at(df[0], (K, I), dF[:, 0:1] * wd)
            np.add.at(df[1], (K, I), dF[:, 1:2] * wd)
            b.ux = b.ux + df[0] * b.dt / (2 * rho)
            b.uz = b.uz + df[1] * b.dt / (2 * rho)
            fib += df
            Ft += dF
        # body: reaction of the marker forces, buoyancy (ref: ibm.cu:383-396),
        # the change of the fluid momentum inside the body, forward Euler
        FdS = Ft * body.dS[:, None]
        r = X - body.X[None]
        Fib = FdS.sum(0)
        Tib = (r[:, 0] * FdS[:, 1] - r[:, 1] * FdS[:, 0]).sum()
        Fb = -(Fib + body.Fib) / 2
        Tb = -(Tib + body.Tib) / 2
        body.Fib, body.Tib = Fib, Tib
        Fb[1] += -(1.0 - self.rho_f / body.rho_s) * body.m * self.g
        xc = (np.arange(b.nx) + 0.5) * b.dz
        zc = (np.arange(b.nz) + 0.5) * b.dz
        XC, ZC = np.meshgrid(xc, zc)
        al = body.fraction(XC, ZC, b.dz) * (b.dz * b.dz)
        P = np.array([(al * b.ux).sum(), (al * b.uz).sum()])
        L = (al * ((XC - body.X[0]) * b.uz - (ZC - body.X[1]) * b.ux)).sum()
        if body.P_in is None:
            body.P_in, body.L_in = P, L
        dt = b.dt
        Uold, omold = body.U.copy(), body.om
        body.U = body.U + (dt * Fb + self.rho_f * (P - body.P_in)) / body.m
        body.om = body.om + (dt * Tb + self.rho_f * (L - body.L_in)) / body.I
        body.X = body.X + dt * (body.U + Uold) / 2
        body.th = body.th + dt * (body.om + omold) / 2
        body.P_in, body.L_in = P, L
