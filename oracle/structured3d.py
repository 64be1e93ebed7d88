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


class Box3D:
    def __init__(self, nx, ny, nz, *, tau=0.55, taus=0.51, g_bouss=1e-5, rho0=1.0, rho_sal=1e-3, dz=1.0,
                 dt=1.0, mrt=True):
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
        self.reg = dz / 1000

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
        """Clamped central differences / (2 dz + dz/1000) along x, y, z."""
        out = []
        for ax, n in ((2, self.nx), (1, self.ny), (0, self.nz)):
            idx = np.arange(n)
            ap = np.take(a, np.minimum(idx + 1, n - 1), axis=ax)
            am = np.take(a, np.maximum(idx - 1, 0), axis=ax)
            # positions of the clamped neighbours: the ghost carries its owner's coordinate
            xp = np.minimum(idx + 1, n - 1) + 0.5
            xm = np.maximum(idx - 1, 0) + 0.5
            den = (xp - xm) * self.dz + self.reg
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

    def step(self, n=1):
        for _ in range(n):
            self._step()

    def _step(self):
        c, c2, dt = self.c, self.c ** 2, self.dt
        p, S, rho, u = self.moments()
        gx, gy, gz = self._grad(rho)
        pc = p * c2 / 3
        F = np.stack([-pc * gx, -pc * gy, -S * self.g_bouss - pc * gz])
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
        self.f = self._stream(fs, E19)
        self.g = self._stream(gs, E7)
        self.F = F
