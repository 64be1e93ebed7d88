"""Synthetic workloads of the benchmark configurations (seeded; no datasets).

`stratified_nonuniform` is the nonuniform-grid two-layer case: 1024 x 256
cells in the x-z plane, uniform in x, tanh-stretched in z
    z(xi) = H zh(xi)/zh(1),  zh(xi) = xi - (gamma/beta) tanh(beta (xi - xi_c)),
beta = 2.0, gamma = 0.812, xi_c so that z(xi_c) = 0.6 H, spacing scaled so the
finest cell equals the lattice spacing (CFL <= 1 on the stretched axis).
Lattice units (dz = dt = 1). D2Q9 MRT with nu = 0.005 (tau = 3 nu + 1/2),
D2Q5 salinity with kappa = 0.0005 (tau_s = kappa/c_s^2 + 1/2), two layers
S = [1 - tanh((z - z_i(x))/delta)]/2 with a 3-cell interface, a 2 % density
difference and an interface tilt of 0.1 H over the tank, g' = 1e-4,
bounce-back walls.
"""
from __future__ import annotations

import numpy as np


def tanh_stretched_axis(n, beta=2.0, gamma=0.812, frac=0.6):
    """Cell centres and widths of n cells on a tanh-clustered axis, finest width 1."""
    xi_e = np.linspace(0.0, 1.0, n + 1)

    def zh(xi, xc):
        return xi - (gamma / beta) * np.tanh(beta * (xi - xc))

    # xi_c such that z(xi_c)/H = frac (bisection; z(xi_c)/H = zh(xi_c)/zh(1))
    lo, hi = 0.0, 1.0
    for _ in range(200):
        xc = 0.5 * (lo + hi)
        if zh(xc, xc) / zh(1.0, xc) < frac:
            lo = xc
        else:
            hi = xc
    xc = 0.5 * (lo + hi)
    edges = zh(xi_e, xc)
    edges = edges - edges[0]
    w = np.diff(edges)
    w = w / w.min()
    e = np.concatenate([[0.0], np.cumsum(w)])
    return 0.5 * (e[1:] + e[:-1]), w, xc


def stratified_nonuniform(nx=1024, nz=256, storage="f32", seed=20261203):
    z, wz, xc = tanh_stretched_axis(nz)
    H = z[-1] + wz[-1] / 2
    x = (np.arange(nx) + 0.5)
    L = float(nx)
    rng = np.random.default_rng(seed)
    zi = 0.6 * H + 0.1 * H * (x / L - 0.5)
    delta = 1.5 * wz.min()  # 3-cell interface at the finest spacing
    S = 0.5 * (1 - np.tanh((z[:, None] - zi[None, :]) / delta))
    S = S + 1e-4 * rng.uniform(-1, 1, S.shape) * (np.abs(z[:, None] - zi[None, :]) < 2 * delta)
    nu, kappa = 0.005, 0.0005
    params = dict(q_scalar=5, geometry="z3", storage=storage, wall="bb", mrt=True, dz=1.0, dt=1.0, z=z, wz=wz,
                  tau=3 * nu + 0.5, taus=3 * kappa + 0.5, rhoL=1.0, rhoH=1.0, phi=1.0, rho_sal=0.02, g_bouss=1e-4,
                  s_ref=0.5)
    meta = dict(nx=nx, nz=nz, spacing_ratio=float(wz.max() / wz.min()), xi_c=float(xc), H=float(H), nu=nu,
                kappa=kappa, g_prime=1e-4, density_difference=0.02)
    return params, S, meta


def lock_exchange_uniform(nx=512, nz=64, seed=20261203):
    """Uniform 512 x 64 lock exchange: S = 1 for x < nx/2 with seeded
    U(-1e-4, 1e-4) noise on the interface columns; g' = 1e-4, nu = 0.01,
    kappa = 0.001 on D2Q5, bounce-back walls."""
    rng = np.random.default_rng(seed)
    x = np.arange(nx)
    S = np.where(x[None, :] < nx // 2, 1.0, 0.0) * np.ones((nz, 1))
    band = np.abs(x + 0.5 - nx / 2) <= 1.0
    S[:, band] += rng.uniform(-1e-4, 1e-4, (nz, band.sum()))
    nu, kappa = 0.01, 0.001
    params = dict(q_scalar=5, geometry="uniform", storage="f32", wall="bb", mrt=True, dz=1.0, dt=1.0,
                  tau=3 * nu + 0.5, taus=3 * kappa + 0.5, rhoL=1.0, rhoH=1.0, phi=1.0, rho_sal=1e-4, g_bouss=1e-4,
                  s_ref=0.5)
    return params, S, dict(nx=nx, nz=nz)


# gravities of the settling-ellipse sweep (lattice units), intended to span
# terminal Reynolds numbers 2 a U / nu of about 1 to 30 for the 20 x 10
# ellipse at nu = 0.02
ELLIPSE_GRAVITIES = (2.5e-6, 1e-5, 4e-5, 1.6e-4)


def settling_ellipse(nx=800, nz=3000, storage="f32", gravity=1e-5, N2=0.0, seed=20261203):
    """An ellipse settling from rest: 800 x 3000 uniform D2Q9 MRT box,
    nu = 0.02, bounce-back walls, semi-axes 20 x 10 cells, 240 markers at
    equal arc length, density ratio 1.1, initial tilt 45 degrees, released at
    (nx/2, 0.85 nz) with a seeded +-2 % jitter of the release point; with
    N2 > 0, a linear salinity stratification N^2 = g' dS/dz on D2Q5
    (kappa = 0.0005). The Boussinesq force -g' S carries the whole
    hydrostatic load, whose pressure range N^2 nz^2 / 2 must stay well below
    c_s^2 = 1/3 for the weakly compressible lattice: N^2 = 1e-6 over 3000
    cells (range 4.5) is beyond it, 1e-8 (0.045) is not. Returns
    (sim params, S0, body dict, meta)."""
    rng = np.random.default_rng(seed)
    nu = 0.02
    S0 = np.zeros((nz, nx))
    qs, gp = 0, 0.0
    if N2 > 0:
        S0 = 1.0 - (np.arange(nz)[:, None] + 0.5) / nz * np.ones((1, nx))
        qs, gp = 5, N2 * nz  # N^2 = g' |dS/dz| with dS/dz = 1/nz
    params = dict(q_scalar=qs, geometry="uniform", storage=storage, wall="bb", mrt=True, dz=1.0, dt=1.0,
                  tau=3 * nu + 0.5, taus=3 * 0.0005 + 0.5, rhoL=1.0, rhoH=1.0, phi=1.0, rho_sal=1e-3, g_bouss=gp,
                  s_ref=0.5)
    j = 1.0 + rng.uniform(-0.02, 0.02, 2)
    body = dict(xc=nx / 2 * j[0], zc=0.85 * nz * j[1], a=20.0, b=10.0, markers=240, theta=np.pi / 4, rho_s=1.1,
                rho_f=1.0, gravity=gravity, iters=3)
    meta = dict(nx=nx, nz=nz, nu=nu, N2=N2)
    return params, S0, body, meta


def centre_clustered_axis(n, ratio=3.0, beta=2.0):
    """Cell centres and widths of n cells tanh-clustered toward the
    centreline: edges x(xi) = xi - (gamma/beta) tanh(beta (xi - 1/2)) on
    xi in [0, 1], gamma chosen (bisection) so that the widest cell is `ratio`
    times the finest, widths scaled so that the finest is one lattice
    spacing (CFL <= 1 on the stretched axis)."""
    xi = np.linspace(0.0, 1.0, n + 1)

    def widths(gamma):
        e = xi - (gamma / beta) * np.tanh(beta * (xi - 0.5))
        return np.diff(e)

    lo, hi = 0.0, 1.0
    for _ in range(200):
        gm = 0.5 * (lo + hi)
        w = widths(gm)
        if w.max() / w.min() < ratio:
            lo = gm
        else:
            hi = gm
    w = widths(0.5 * (lo + hi))
    w = w / w.min()
    e = np.concatenate([[0.0], np.cumsum(w)])
    return 0.5 * (e[1:] + e[:-1]), w


def clustered_box_3d(nx=160, ny=160, nz=640, ratio=3.0, seed=20261203):
    """The 3-D configuration's box without its body: D3Q19 MRT + D3Q7 on
    nx x ny x nz cells, x and y tanh-clustered toward the centreline (spacing
    ratio 3), z uniform, a linear salinity stratification S = 1 - z/H with
    seeded 1e-4 noise, tau = 0.55, tau_s = 0.52, Boussinesq g' = 1e-5 with
    rho = 1 + 1e-3 S, bounce-back walls. Returns (Sim3D keyword arguments, S0)."""
    x, wx = centre_clustered_axis(nx, ratio)
    y, wy = centre_clustered_axis(ny, ratio)
    rng = np.random.default_rng(seed)
    zz = np.broadcast_to((np.arange(nz) + 0.5)[:, None, None] / nz, (nz, ny, nx))
    S0 = 1.0 - zz + 1e-4 * rng.uniform(-1, 1, (nz, ny, nx))
    kw = dict(tau=0.55, taus=0.52, rho_sal=1e-3, g_bouss=1e-5, x=x, wx=wx, y=y, wy=wy, ns=3)
    return kw, S0


def falling_sphere_3d(kw, nx, ny, nz, seed=20261203, gravity=2e-5):
    """The 3-D configuration's falling sphere for a box built by
    clustered_box_3d (kw: its keyword arguments): diameter 16 finest cells
    (radius 8 in the finest spacing), about 800 markers on a Fibonacci
    lattice, density ratio 1.5, released from rest at 0.8 of the height on
    the centreline with a seeded lateral offset of at most one cell, lattice
    gravity 2e-5 (one value of the sweep). Returns Sim3D.attach_sphere
    keyword arguments."""
    rng = np.random.default_rng(seed)
    x = kw.get("x", np.arange(nx) + 0.5)
    y = kw.get("y", np.arange(ny) + 0.5)
    off = rng.uniform(-1.0, 1.0, 2)
    xc = 0.5 * (x[nx // 2 - 1] + x[nx // 2]) + off[0]
    yc = 0.5 * (y[ny // 2 - 1] + y[ny // 2]) + off[1]
    return dict(xc=float(xc), yc=float(yc), zc=0.8 * nz, radius=8.0, markers=804, rho_s=1.5, rho_f=1.0,
                gravity=gravity, iters=3)
