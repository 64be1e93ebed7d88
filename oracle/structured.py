"""ORACLE -- test infrastructure only. FP64 numpy restatement of one
LockExchange-ordered step on a rectangular x-z box, written as whole-field
array operations (independent of the CUDA tile kernel it checks).

Step (ref: LockExchange/LockExchange.cu:220-236):
  feq(p*, u), F = buoyancy - p* c^2/3 grad(rho), Fk    (function/collision.cu:3-14,57-112)
  MRT (or BGK) collision of f                          (collision.cu:115-165)
  regularised collision of the scalar g                (collision.cu:167-188)
  conservative interpolated streaming of f and g       (function/adv.cu:50-257,
                                                        set_bound.cu:164-183, propagation.cu)
  S = sum g, p* = sum f, u = sum e f + F dt / 2 rho    (collision.cu:225-257)

Phase-field mode (phase_field=True): the scalar lattice carries the
Allen-Cahn order parameter phi instead of salinity, in the reference's
two-phase step order (RTinstability/RTinstability.cu:177-206):
  rho = rhoL + (rhoH - rhoL) phi; F = mu grad(phi) - rho g e_z - p* c^2/3 grad(rho)
  with mu = 4 beta phi (phi - 1)(phi - 1/2) - kappa lap(phi)  (collision.cu:57-112, Boussi_flag off)
  conservative Allen-Cahn collision of g with the d(phi u)/dt term (collision.cu:190-223)
  phi = sum g                                                   (collision.cu:225-236)

On the reference's own layouts it is pinned against the oracle's kernel
chain (tests/test_structured_oracle.py); it extends the same rules to an
interpolated z axis, the 3-point upwind-biased quadratic stencil and the
D2Q5 scalar lattice, which the reference does not have.
"""
from __future__ import annotations

import numpy as np

EX9 = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
EZ9 = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
W5 = np.array([1 / 3] + [1 / 6] * 4)
KINV9 = [0, 3, 4, 1, 2, 7, 8, 5, 6]

GEOS = {"uniform": (None, 1), "x5": (0, 5), "x3": (0, 3), "z5": (1, 5), "z3": (1, 3)}


def mirror(k, axis):
    ex, ez = EX9[k], EZ9[k]
    if axis == 0:
        ex = -ex
    else:
        ez = -ez
    for q in range(9):
        if EX9[q] == ex and EZ9[q] == ez:
            return q
    raise ValueError


def stencil_weights(X, D, dz, ns):
    """W[s, j, m], fin scale [s, j], fout scale [j] of the flux form along one axis."""
    n = len(X)
    W = np.zeros((2, n, ns))
    sin = np.zeros((2, n))
    sout = dz / np.asarray(D, float)
    h = ns // 2
    for j in range(n):
        for s, sg in ((0, 1), (1, -1)):
            xa = X[j] + sg * (D[j] - dz) / 2
            nodes = [X[min(max(j + sg * (m - h), 0), n - 1)] for m in range(ns)]
            # nodes past a wall sit one lattice spacing beyond their inner neighbour
            for m in range(h - 1, -1, -1):
                nodes[m] = min(nodes[m], nodes[m + 1] - dz) if sg > 0 else max(nodes[m], nodes[m + 1] + dz)
            for m in range(h + 1, ns):
                nodes[m] = max(nodes[m], nodes[m - 1] + dz) if sg > 0 else min(nodes[m], nodes[m - 1] - dz)
            for a in range(ns):
                v = 1.0
                for b in range(ns):
                    if b != a:
                        v *= (xa - nodes[b]) / (nodes[a] - nodes[b])
                W[s, j, a] = v
            sin[s, j] = dz / D[min(max(j + sg, 0), n - 1)]
    return W, sin, sout


def _dir(ex, ez):
    return [q for q in range(9) if EX9[q] == ex and EZ9[q] == ez][0]


def slip_partner(k, L, R, B, T):
    """(neighbour direction, population) a specular wall reflects into the
    ghost of a cell whose source for direction k lies outside the box
    (ref: function/set_bound.cu:40-73)."""
    cx, cz = EX9[k], EZ9[k]
    if (R and cx == -1) or (L and cx == 1):
        cx = 0
    if (T and cz == -1) or (B and cz == 1):
        cz = 0
    if cx != 0 and cz == 0 and EZ9[k] != 0:  # reflected off a z wall
        return (3 if cx > 0 else 1), _dir(EX9[k], -EZ9[k])
    if cz != 0 and cx == 0 and EX9[k] != 0:  # reflected off an x wall
        return (4 if cz > 0 else 2), _dir(-EX9[k], EZ9[k])
    return 0, KINV9[k]


class Box:
    def __init__(self, nx, nz, *, q_scalar=5, geometry="uniform", wall="bb", mrt=True, dz=1.0, dt=1.0, x=None,
                 z=None, wx=None, wz=None, tau=0.53, taus=0.503, rhoL=1.0, rhoH=1.0, phi=1.0, rho_sal=0.0,
                 g_bouss=1e-4, M=None, Minv=None, S=None, phase_field=False, sigma=0.0, pf_width=4.0,
                 gravity=0.0):
        self.nx, self.nz, self.qs = nx, nz, q_scalar
        self.pf, self.sigma, self.pfw, self.grav = phase_field, sigma, pf_width, gravity
        self.rhoL, self.rhoH = rhoL, rhoH
        self.axis, self.ns = GEOS[geometry]
        self.wall, self.mrt = wall, mrt
        self.dz, self.dt, self.c = dz, dt, dz / dt
        self.X = np.asarray(x if x is not None else (np.arange(nx) + 0.5) * dz, float)
        self.Z = np.asarray(z if z is not None else (np.arange(nz) + 0.5) * dz, float)
        self.DX = np.asarray(wx if wx is not None else np.full(nx, dz), float)
        self.DZ = np.asarray(wz if wz is not None else np.full(nz, dz), float)
        self.tau, self.taus = tau, taus
        self.rho0 = rhoL + (rhoH - rhoL) * phi
        self.rho_sal, self.g_bouss = rho_sal, g_bouss
        if mrt:
            Sv = np.array(S, float).copy()
            Sv[7] = Sv[8] = 0.0
            self.MM = np.asarray(Minv) @ np.diag(Sv) @ np.asarray(M)
            self.Ps = np.asarray(Minv)[:, 7:9] @ np.asarray(M)[7:9, :]
        if self.axis is not None:
            A = (self.X, self.DX) if self.axis == 0 else (self.Z, self.DZ)
            self.W, self.sin, self.sout = stencil_weights(A[0], A[1], dz, self.ns)
        reg = dz / 1000
        cl = lambda a, i: a[np.clip(i, 0, len(a) - 1)]
        self.gix = 1 / (cl(self.X, np.arange(nx) + 1) - cl(self.X, np.arange(nx) - 1) + reg)
        self.giz = 1 / (cl(self.Z, np.arange(nz) + 1) - cl(self.Z, np.arange(nz) - 1) + reg)
        self.f = np.zeros((9, nz, nx))
        self.g = np.zeros((max(q_scalar, 1), nz, nx))
        self.S = np.zeros((nz, nx))
        self.ux = np.zeros((nz, nx))
        self.uz = np.zeros((nz, nx))
        self.old = np.zeros((2, nz, nx))  # phase field: phi u, phi w of the previous step
        self.fext = np.zeros((2, nz, nx))  # external force density (immersed boundary), added to F

    # ------------------------------------------------------------------ pieces
    def _interp(self, fs, s):
        """I[j] of every cell along the axis for one population field fs[nz, nx]."""
        n = fs.shape[1] if self.axis == 0 else fs.shape[0]
        sg = 1 if s == 0 else -1
        h = self.ns // 2
        out = np.zeros_like(fs)
        for m in range(self.ns):
            idx = np.clip(np.arange(n) + sg * (m - h), 0, n - 1)
            w = self.W[s, :, m]
            if self.axis == 0:
                out += w[None, :] * fs[:, idx]
            else:
                out += w[:, None] * fs[idx, :]
        return out

    def _ftmp(self, fs, qn):
        """The reference's post-set_tmp field of every direction (ref: adv.cu:234-244)."""
        if self.axis is None:
            return fs.copy()
        out = np.empty_like(fs)
        e = EX9 if self.axis == 0 else EZ9
        for k in range(qn):
            a = e[k]
            if a == 0:
                out[k] = fs[k]
                continue
            s = 0 if a > 0 else 1
            I = self._interp(fs[k], s)
            if self.axis == 0:
                fin = I * self.sin[s][None, :]
                fout = I * self.sout[None, :]
                km = mirror(k, 0)
                Im = self._interp(fs[km], 1 - s) * self.sout[None, :]
                shifted_f = np.roll(fs[k], -a, axis=1)
                shifted_o = np.roll(fout, -a, axis=1)
                edge = self.nx - 1 if a > 0 else 0
                shifted_f[:, edge] = fs[km][:, edge]
                shifted_o[:, edge] = Im[:, edge]
            else:
                fin = I * self.sin[s][:, None]
                fout = I * self.sout[:, None]
                km = mirror(k, 1)
                Im = self._interp(fs[km], 1 - s) * self.sout[:, None]
                shifted_f = np.roll(fs[k], -a, axis=0)
                shifted_o = np.roll(fout, -a, axis=0)
                edge = self.nz - 1 if a > 0 else 0
                shifted_f[edge, :] = fs[km][edge, :]
                shifted_o[edge, :] = Im[edge, :]
            out[k] = shifted_f + (fin - shifted_o)
        return out

    def _stream(self, fs, qn):
        t = self._ftmp(fs, qn)
        nz, nx = self.nz, self.nx
        new = np.empty_like(fs)
        zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
        for k in range(qn):
            sx, sz = xx - EX9[k], zz - EZ9[k]
            inside = (sx >= 0) & (sx < nx) & (sz >= 0) & (sz < nz)
            v = np.empty((nz, nx))
            v[inside] = t[k][sz[inside], sx[inside]]
            out_i = np.argwhere(~inside)
            for (iz, ix) in out_i:
                if self.wall == "bb":
                    v[iz, ix] = t[KINV9[k]][iz, ix]
                else:
                    L, R, B, T = ix == 0, ix == nx - 1, iz == 0, iz == nz - 1
                    nb, kk = slip_partner(k, L, R, B, T) if qn == 9 else (0, KINV9[k])
                    v[iz, ix] = t[kk][iz + EZ9[nb], ix + EX9[nb]]
            new[k] = v
        return new

    def rho_of(self, S):
        """Density from the scalar field: the mixture rhoL + (rhoH - rhoL) phi
        (phase field) or rho0 + rho_sal S (salinity) (ref: collision.cu:251)."""
        if self.pf:
            return self.rhoL + (self.rhoH - self.rhoL) * S
        return self.rho0 + self.rho_sal * S

    # ------------------------------------------------------------------ step
    def step(self, n=1):
        for _ in range(n):
            self._step()

    def _step(self):
        c, c2, dt = self.c, self.c ** 2, self.dt
        f, S, u, w = self.f, self.S, self.ux, self.uz
        p = f.sum(0)
        rho = self.rho_of(S)
        xi = np.arange(self.nx)
        zi = np.arange(self.nz)
        rxp = rho[:, np.minimum(xi + 1, self.nx - 1)]
        rxm = rho[:, np.maximum(xi - 1, 0)]
        rzp = rho[np.minimum(zi + 1, self.nz - 1), :]
        rzm = rho[np.maximum(zi - 1, 0), :]
        pc = p * c2 / 3
        Fx = -pc * (rxp - rxm) * self.gix[None, :]
        Fz = -pc * (rzp - rzm) * self.giz[:, None]
        if self.pf:
            # surface tension mu grad(phi) (chemical potential of the double
            # well) and the weight of the mixture (ref: collision.cu:65-78)
            sxp = S[:, np.minimum(xi + 1, self.nx - 1)]
            sxm = S[:, np.maximum(xi - 1, 0)]
            szp = S[np.minimum(zi + 1, self.nz - 1), :]
            szm = S[np.maximum(zi - 1, 0), :]
            dpx = (sxp - sxm) * self.gix[None, :]
            dpz = (szp - szm) * self.giz[:, None]
            lap = (sxp - 2 * S + sxm) / self.DX[None, :] ** 2 + (szp - 2 * S + szm) / self.DZ[:, None] ** 2
            beta, kap = 12 * self.sigma / self.pfw, 1.5 * self.sigma * self.pfw
            mu = 4 * beta * S * (S - 1) * (S - 0.5) - kap * lap
            Fx = Fx + mu * dpx
            Fz = Fz + mu * dpz - rho * self.grav
        else:
            Fz = Fz - S * self.g_bouss
        Fx = Fx + self.fext[0]
        Fz = Fz + self.fext[1]
        eu = c * (EX9[:, None, None] * u[None] + EZ9[:, None, None] * w[None]) / c2
        us = (u * u + w * w) / c2
        feq = W9[:, None, None] * (p[None] + 3 * eu + 4.5 * eu ** 2 - 1.5 * us[None])
        Fk = W9[:, None, None] * c * (EX9[:, None, None] * Fx[None] + EZ9[:, None, None] * Fz[None]) * dt / (
            rho[None] * c2 / 3)
        d = f - feq + Fk / 2
        if self.mrt:
            D = d.reshape(9, -1)
            fs = f - (self.MM @ D + (self.Ps @ D) / self.tau).reshape(f.shape) + Fk
        else:
            fs = f - d / self.tau + Fk
        qs = self.qs
        if qs:
            w_ = W5 if qs == 5 else W9
            eq = c * (EX9[:qs, None, None] * u[None] + EZ9[:qs, None, None] * w[None]) / c2
            shape = 1 + 3 * eq if qs == 5 else 1 + 3 * eq + 4.5 * eq ** 2 - 1.5 * us[None]
            geq = w_[:, None, None] * S[None] * shape
            if self.pf:
                # conservative Allen-Cahn collision (ref: collision.cu:190-223):
                # g* = g - (g - geq)/tau_phi + (tau_phi - 1/2)/tau_phi Fp, with
                # Fp_k = dt w_k [(1 - 4 (phi - 1/2)^2)/W c e.grad(phi)/|grad(phi)|
                #                + 3 e.d(phi u)/dt / c]
                nab = (S * u - self.old[0]) / dt, (S * w - self.old[1]) / dt
                self.old = np.stack([S * u, S * w])
                nrm = np.sqrt(dpx ** 2 + dpz ** 2 + 1e-8)
                ed = EX9[:qs, None, None] * dpx[None] + EZ9[:qs, None, None] * dpz[None]
                en = EX9[:qs, None, None] * nab[0][None] + EZ9[:qs, None, None] * nab[1][None]
                Fp = dt * w_[:, None, None] * ((1 - 4 * (S - 0.5) ** 2)[None] / self.pfw * c * ed / nrm[None]
                                               + 3 * en / c)
                ts = self.taus
                gs = self.g - (self.g - geq) / ts + (ts - 0.5) / ts * Fp
            else:
                ne = self.g - geq
                jx = (ne * (c * EX9[:qs, None, None])).sum(0)
                jz = (ne * (c * EZ9[:qs, None, None])).sum(0)
                gs = geq + (1 - 1 / self.taus) * w_[:, None, None] * 3 * (
                    jx[None] * c * EX9[:qs, None, None] + jz[None] * c * EZ9[:qs, None, None]) / c2
            self.g = self._stream(gs, qs)
            S = self.g.sum(0)
        self.f = self._stream(fs, 9)
        p2 = self.f.sum(0)
        rho2 = self.rho_of(S)
        h = dt / (2 * rho2)
        self.ux = (self.f * (c * EX9[:, None, None])).sum(0) + Fx * h
        self.uz = (self.f * (c * EZ9[:, None, None])).sum(0) + Fz * h
        self.S = S
        self.p = p2
