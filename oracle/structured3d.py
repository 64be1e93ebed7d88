"""ORACLE -- test infrastructure only. FP64 numpy restatement of one step of
the 3-D path on a rectangular box with a uniform lattice: D3Q19 flow with
MRT collision (d'Humieres moment basis; the five shear moments relax with
1/tau, all others with rate 1 -- the reference's unit-rate S file applied
to D3Q19), Boussinesq buoyancy and the pressure-gradient force of the
reference's Force kernel, a D3Q7 passive salinity with the regularised
collision of col_g_reg, halfway bounce-back on all six faces, in the
reference's step order (ref: LockExchange/LockExchange.cu:220-236;
function/collision.cu:3-188,238-257; propagation.cu; set_bound.cu:164-183):

  p* = sum f, S = sum g, u = c sum e f + F_prev dt / 2 rho  (collision.cu:238-257)
  F = -S g' e_z - p* c^2/3 grad(rho)                           (collision.cu:57-112)
  f* = f - Minv diag(s) M (f - feq + Fk/2) + Fk               (collision.cu:115-150)
  g* = geq + (1 - 1/tau_s) w_k e_k.j / cs^2                   (collision.cu:167-188, D3Q7)
  f(x) <- f*(x - e_k), bounce-back where x - e_k is outside

Velocity orders follow the reference's D3Q27 (ref: function/basic.cu:88-97):
D3Q19 is its first 19 directions, D3Q7 its first 7. D3Q7 weights 1/4, 1/8
(cs^2 = 1/4), equilibrium w S (1 + 4 e.u/c).

The reference has no D3Q19/D3Q7 path, so parity for this mode is against
this restatement (the same rules as the reference's D3Q27 kernels, on the
D3Q19 subset), not against the reference build.

Stretched x and y axes (x, wx / y, wy given; z stays uniform): streaming is
the reference's conservative interpolated flux form (ref: function/adv.cu:
50-147,176-257) with an ns-point Lagrange stencil per axis (5 = the
reference's, 3 = quadratic upwind), weights and clamped nodes as
set_posl_x/Lagrange_interpolation give them:
  * populations moving along x only (in-plane), or y only: the 1-D flux form
    of set_out's first two loops, ftmp(c) = f*(c+a) + fin(c) - fout(c+a),
    fin = I dz/D(c+a), fout = I dz/D;
  * populations moving along an xy diagonal: set_out's corner-transport
    form, fout(i) = fx dz/DX + fy dz/DY - fxy dz^2/(DX DY) and the three
    fin contributions of cells i, i+x, i+y (adv.cu:141-144), so that
    ftmp(c) = f*(d) + fin(c) - fout(d) with d = c + e_xy;
  * the z component is an exact shift, then f(c) = ftmp(c - e) (propagation).
Walls (bounce-back on all faces): interpolation nodes past a wall take the
owner's value (set_wall_f); a ghost cell across an x or y wall is the mirror
image of its owner -- its populations, and the flux quantities fx, fy, fxy
built from them, are the owner's for the population mirrored across that
wall (set_wall_f_inv's rule for the in-plane mirror, applied to every
quantity the flux form reads); a source outside the box bounces back,
f(c, k) = ftmp(c, -k). In the interior the diagonal form equals the tensor
product of the two 1-D flux-form operators.
"""
from __future__ import annotations

import numpy as np

E27 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [-1, 0, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                [1, 1, 0], [1, -1, 0], [-1, 1, 0], [-1, -1, 0], [1, 0, 1], [1, 0, -1], [-1, 0, 1], [-1, 0, -1],
                [0, 1, 1], [0, 1, -1], [0, -1, 1], [0, -1, -1]])
E19 = E27[:19]
E7 = E27[:7]
W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
W7 = np.array([1 / 4] + [1 / 8] * 6)
KINV19 = [int(np.where((E19 == -e).all(1))[0][0]) for e in E19]


def d3q19_mrt():
    """d'Humieres D3Q19 moment matrix (rows: rho, e, eps, jx, qx, jy, qy, jz,
    qz, 3pxx, 3pixx, pww, piww, pxy, pyz, pxz, mx, my, mz), its inverse and the
    relaxation rates with the shear rows (9, 11, 13, 14, 15) marked 0 (they
    relax with 1/tau)."""
    ex, ey, ez = E19[:, 0].astype(float), E19[:, 1].astype(float), E19[:, 2].astype(float)
    e2 = ex * ex + ey * ey + ez * ez
    rows = [np.ones(19), 19 * e2 - 30, (21 * e2 * e2 - 53 * e2 + 24) / 2,
            ex, (5 * e2 - 9) * ex, ey, (5 * e2 - 9) * ey, ez, (5 * e2 - 9) * ez,
            3 * ex * ex - e2, (3 * e2 - 5) * (3 * ex * ex - e2), ey * ey - ez * ez, (3 * e2 - 5) * (ey * ey - ez * ez),
            ex * ey, ey * ez, ex * ez,
            (ey * ey - ez * ez) * ex, (ez * ez - ex * ex) * ey, (ex * ex - ey * ey) * ez]
    M = np.stack(rows)
    S = np.ones(19)
    S[[9, 11, 13, 14, 15]] = 0.0
    return M, np.linalg.inv(M), S


def mirror3(k, ax, ay):
    """Direction of the population mirrored across an x wall (ax), a y wall
    (ay) or both."""
    e = E19[k].copy()
    if ax:
        e[0] = -e[0]
    if ay:
        e[1] = -e[1]
    return int(np.where((E19 == e).all(1))[0][0])


class Box3D:
    def __init__(self, nx, ny, nz, *, tau=0.55, taus=0.51, g_bouss=1e-5, rho0=1.0, rho_sal=1e-3, dz=1.0,
                 dt=1.0, mrt=True, x=None, wx=None, y=None, wy=None, ns=3):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.tau, self.taus, self.g_bouss, self.rho0, self.rho_sal = tau, taus, g_bouss, rho0, rho_sal
        self.dz, self.dt, self.c = dz, dt, dz / dt
        self.mrt = mrt
        M, Minv, S = d3q19_mrt()
        self.M, self.Minv, self.S = M, Minv, S
        shape = (nz, ny, nx)
        self.f = np.zeros((19,) + shape)
        self.g = np.zeros((7,) + shape)
        self.F = np.zeros((3,) + shape)  # force of the previous step
        self.fext = np.zeros((3,) + shape)  # external force density (immersed boundary), added to F
        self.reg = dz / 1000
        self.stretched = x is not None or y is not None
        self.X = np.asarray(x if x is not None else (np.arange(nx) + 0.5) * dz, float)
        self.DX = np.asarray(wx if wx is not None else np.full(nx, dz), float)
        self.Y = np.asarray(y if y is not None else (np.arange(ny) + 0.5) * dz, float)
        self.DY = np.asarray(wy if wy is not None else np.full(ny, dz), float)
        self.ns = ns
        if self.stretched:
            from oracle.structured import stencil_weights

            self.Wx, self.sinx, self.soutx = stencil_weights(self.X, self.DX, dz, ns)
            self.Wy, self.siny, self.souty = stencil_weights(self.Y, self.DY, dz, ns)

    # the three macroscopic fields the kernel forms at the start of a step
    def moments(self):
        c = self.c
        p = self.f.sum(0)
        S = self.g.sum(0)
        rho = self.rho0 + self.rho_sal * S
        h = self.dt / (2 * rho)
        u = [c * np.tensordot(E19[:, a].astype(float), self.f, 1) + self.F[a] * h for a in range(3)]
        return p, S, rho, u

    def _grad(self, a):
        """Clamped central differences / (x_{i+1} - x_{i-1} + dz/1000) along x, y, z."""
        out = []
        zc = (np.arange(self.nz) + 0.5) * self.dz
        for ax, n, pos in ((2, self.nx, self.X), (1, self.ny, self.Y), (0, self.nz, zc)):
            idx = np.arange(n)
            ap = np.take(a, np.minimum(idx + 1, n - 1), axis=ax)
            am = np.take(a, np.maximum(idx - 1, 0), axis=ax)
            # positions of the clamped neighbours: the ghost carries its owner's coordinate
            den = pos[np.minimum(idx + 1, n - 1)] - pos[np.maximum(idx - 1, 0)] + self.reg
            sh = [1, 1, 1]
            sh[ax] = n
            out.append((ap - am) / den.reshape(sh))
        return out

    def _stream(self, fs, E):
        q = len(E)
        kinv = [int(np.where((E == -e).all(1))[0][0]) for e in E]
        nz, ny, nx = fs.shape[1:]
        new = np.empty_like(fs)
        for k in range(q):
            ex, ey, ez = E[k]
            src = np.roll(fs[k], (ez, ey, ex), axis=(0, 1, 2))  # src[x] = fs[x - e]
            # cells whose source x - e lies outside take their own bounced population
            zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
            out = ((xx - ex < 0) | (xx - ex >= nx) | (yy - ey < 0) | (yy - ey >= ny) | (zz - ez < 0) |
                   (zz - ez >= nz))
            src[out] = fs[kinv[k]][out]
            new[k] = src
        return new

    # ---------------------------------------------------------------- stretched x, y
    def _interp(self, a, s, axis):
        """I of every cell along x (axis 2) or y (axis 1) with clamped nodes;
        s = 0 for a population moving in +, 1 in -."""
        W = self.Wx if axis == 2 else self.Wy
        n = a.shape[axis]
        sg = 1 if s == 0 else -1
        h = self.ns // 2
        out = np.zeros_like(a)
        for m in range(self.ns):
            idx = np.clip(np.arange(n) + sg * (m - h), 0, n - 1)
            sh = [1, 1, 1]
            sh[axis] = n
            out += W[s, :, m].reshape(sh) * np.take(a, idx, axis=axis)
        return out

    def _ftmp_axis(self, fs, k, axis, E):
        """1-D flux form along x (axis 2) or y (axis 1) for population k."""
        comp = 0 if axis == 2 else 1
        a = int(E[k][comp])
        s = 0 if a > 0 else 1
        sin = self.sinx if axis == 2 else self.siny
        sout = self.soutx if axis == 2 else self.souty
        n = fs.shape[axis + 1]
        sh = [1, 1, 1]
        sh[axis] = n
        I = self._interp(fs[k], s, axis)
        fin = I * sin[s].reshape(sh)
        fout = I * sout.reshape(sh)
        km = int(np.where((E == E[k] * np.array([-1 if comp == 0 else 1, -1 if comp == 1 else 1, 1])).all(1))[0][0])
        Im = self._interp(fs[km], 1 - s, axis) * sout.reshape(sh)
        shifted_f = np.roll(fs[k], -a, axis=axis)
        shifted_o = np.roll(fout, -a, axis=axis)
        edge = n - 1 if a > 0 else 0
        sl = [slice(None)] * 3
        sl[axis] = edge
        shifted_f[tuple(sl)] = fs[km][tuple(sl)]
        shifted_o[tuple(sl)] = Im[tuple(sl)]
        return shifted_f + (fin - shifted_o)

    def _ftmp_diag(self, fs, k):
        """Corner-transport flux form of an xy-diagonal population k with
        mirror-image ghosts across the x and y walls."""
        nz, ny, nx = fs.shape[1:]
        sx, sy = int(E19[k][0]), int(E19[k][1])
        dz = self.dz

        def quantities(kk):
            ex, ey = int(E19[kk][0]), int(E19[kk][1])
            fx = self._interp(fs[kk], 0 if ex > 0 else 1, 2)
            fy = self._interp(fs[kk], 0 if ey > 0 else 1, 1)
            fxy = self._interp(self._interp(fs[kk], 0 if ex > 0 else 1, 2), 0 if ey > 0 else 1, 1)
            return fs[kk], fx, fy, fxy

        def extend(q, qx, qy, qxy):
            """q on (nz, ny + 2, nx + 2) with mirror ghosts."""
            out = np.zeros((nz, ny + 2, nx + 2))
            out[:, 1:-1, 1:-1] = q
            out[:, 1:-1, 0], out[:, 1:-1, -1] = qx[:, :, 0], qx[:, :, -1]
            out[:, 0, 1:-1], out[:, -1, 1:-1] = qy[:, 0, :], qy[:, -1, :]
            out[:, 0, 0], out[:, 0, -1] = qxy[:, 0, 0], qxy[:, 0, -1]
            out[:, -1, 0], out[:, -1, -1] = qxy[:, -1, 0], qxy[:, -1, -1]
            return out

        base = quantities(k)
        mx, my, mxy = (quantities(mirror3(k, 1, 0)), quantities(mirror3(k, 0, 1)), quantities(mirror3(k, 1, 1)))
        F, FX, FY, FXY = (extend(base[i], mx[i], my[i], mxy[i]) for i in range(4))
        yy, xx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        # extended indices of c, c + sx, c + sy, d = c + sx + sy
        cy, cx = yy + 1, xx + 1
        ax = dz / self.DX[np.clip(xx + sx, 0, nx - 1)]
        ay = dz / self.DY[np.clip(yy + sy, 0, ny - 1)]
        g = lambda A, oy, ox: A[:, cy + oy, cx + ox]
        fin = (ax * ay) * g(FXY, 0, 0) + ay * (g(FY, 0, sx) - ax * g(FXY, 0, sx)) + ax * (g(FX, sy, 0) - ay * g(FXY, sy, 0))
        fout = ax * g(FX, sy, sx) + ay * g(FY, sy, sx) - (ax * ay) * g(FXY, sy, sx)
        return g(F, sy, sx) + (fin - fout)

    def _stream_stretched(self, fs, E):
        q = len(E)
        kinv = [int(np.where((E == -e).all(1))[0][0]) for e in E]
        t = np.empty_like(fs)
        for k in range(q):
            ex, ey = int(E[k][0]), int(E[k][1])
            if ex == 0 and ey == 0:
                t[k] = fs[k]
            elif ey == 0:
                t[k] = self._ftmp_axis(fs, k, 2, E)
            elif ex == 0:
                t[k] = self._ftmp_axis(fs, k, 1, E)
            else:
                t[k] = self._ftmp_diag(fs, k)
        nz, ny, nx = fs.shape[1:]
        zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        new = np.empty_like(fs)
        for k in range(q):
            ex, ey, ez = E[k]
            sx, sy, sz = xx - ex, yy - ey, zz - ez
            inside = (sx >= 0) & (sx < nx) & (sy >= 0) & (sy < ny) & (sz >= 0) & (sz < nz)
            v = t[kinv[k]].copy()  # bounce-back where the source lies outside the box
            v[inside] = t[k][sz[inside], sy[inside], sx[inside]]
            new[k] = v
        return new

    def step(self, n=1):
        for _ in range(n):
            self._step()

    def _step(self):
        c, c2, dt = self.c, self.c ** 2, self.dt
        p, S, rho, u = self.moments()
        gx, gy, gz = self._grad(rho)
        pc = p * c2 / 3
        F = np.stack([-pc * gx, -pc * gy, -S * self.g_bouss - pc * gz]) + self.fext
        uc = [a / c for a in u]
        eu = sum(E19[:, a].astype(float)[:, None, None, None] * uc[a][None] for a in range(3))
        us = sum(a * a for a in uc)
        feq = W19[:, None, None, None] * (p[None] + 3 * eu + 4.5 * eu ** 2 - 1.5 * us[None])
        ef = sum(E19[:, a].astype(float)[:, None, None, None] * F[a][None] for a in range(3))
        Fk = W19[:, None, None, None] * c * ef * dt / (rho[None] * c2 / 3)
        d = self.f - feq + Fk / 2
        if self.mrt:
            s = self.S.copy()
            s[s == 0] = 1 / self.tau
            D = d.reshape(19, -1)
            fs = self.f - (self.Minv @ (s[:, None] * (self.M @ D))).reshape(d.shape) + Fk
        else:
            fs = self.f - d / self.tau + Fk
        # D3Q7 regularised scalar collision, cs^2 = 1/4
        eu7 = sum(E7[:, a].astype(float)[:, None, None, None] * uc[a][None] for a in range(3))
        geq = W7[:, None, None, None] * S[None] * (1 + 4 * eu7)
        ne = self.g - geq
        j = [np.tensordot(E7[:, a].astype(float), ne, 1) for a in range(3)]
        ej = sum(E7[:, a].astype(float)[:, None, None, None] * j[a][None] for a in range(3))
        gs = geq + (1 - 1 / self.taus) * W7[:, None, None, None] * 4 * ej
        if self.stretched:
            self.f = self._stream_stretched(fs, E19)
            self.g = self._stream_stretched(gs, E7)
        else:
            self.f = self._stream(fs, E19)
            self.g = self._stream(gs, E7)
        self.F = F
