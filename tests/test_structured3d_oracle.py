"""The FP64 3-D oracle (oracle/structured3d.py): its MRT reduces to BGK when
every rate is 1/tau, the d'Humieres basis is orthogonal, the rest state is
kept exactly, and bounce-back conserves p* and S."""
import numpy as np

from oracle.structured3d import Box3D, E19, W19, W7, d3q19_mrt


def _state(b, seed):
    rng = np.random.default_rng(seed)
    nz, ny, nx = b.nz, b.ny, b.nx
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    S = 0.5 + 0.3 * np.sin(2 * np.pi * xx / nx) * np.cos(np.pi * zz / nz)
    u = [1e-3 * np.sin(2 * np.pi * zz / nz + a) for a in (0.0, 1.0, 2.0)]
    eu = sum(E19[:, a][:, None, None, None] * u[a][None] for a in range(3))
    us = sum(a * a for a in u)
    f = W19[:, None, None, None] * (3 * eu + 4.5 * eu ** 2 - 1.5 * us[None])
    f += 1e-5 * W19[:, None, None, None] * rng.standard_normal(f.shape)
    g = W7[:, None, None, None] * S[None] * (1 + 4 * sum(E19[:7, a][:, None, None, None] * u[a][None]
                                                         for a in range(3)))
    return f, g


def test_basis_orthogonal():
    M, Minv, S = d3q19_mrt()
    G = M @ M.T
    assert np.allclose(G - np.diag(np.diag(G)), 0)
    assert np.allclose(M @ Minv, np.eye(19))
    # shear row norms used by the fused kernel's closed form
    assert np.allclose(np.diag(G)[[9, 11, 13, 14, 15]], [36, 12, 4, 4, 4])


def test_mrt_with_uniform_rates_is_bgk():
    a = Box3D(8, 6, 5, tau=0.7, g_bouss=1e-4, rho_sal=1e-3)
    b = Box3D(8, 6, 5, tau=0.7, g_bouss=1e-4, rho_sal=1e-3, mrt=False)
    f, g = _state(a, 1)
    for x in (a, b):
        x.f, x.g = f.copy(), g.copy()
    a.S = np.full(19, 1 / 0.7)  # every moment at 1/tau
    a.step(5)
    b.step(5)
    assert np.abs(a.f - b.f).max() <= 1e-14


def test_rest_state_exact():
    b = Box3D(6, 5, 4, g_bouss=0.0)
    b.g[:] = (W7 * 0.3)[:, None, None, None]
    b.step(5)
    assert not np.any(b.f)
    assert np.abs(b.g.sum(0) - 0.3).max() <= 1e-15


def test_bounce_back_conserves_mass():
    b = Box3D(10, 8, 6, g_bouss=1e-4, rho_sal=1e-3)
    b.f, b.g = _state(b, 2)
    p0, s0 = b.f.sum(), b.g.sum()
    b.step(20)
    assert abs(b.f.sum() - p0) <= 1e-12 and abs(b.g.sum() - s0) <= 1e-12 * s0
