"""The fused 3-D step on stretched x and y axes (ipcu_sim3d_create_stretched:
D3Q19 MRT + D3Q7, the conservative interpolated flux form along x and y,
corner transport for the xy diagonals) against
  * the FP64 oracle with the same rules (oracle/structured3d.py, stretched
    mode), rel-L2 <= 1e-5 on u, S and p*, for the 3-point and the reference's
    5-point stencil, on clustered axes (spacing ratio 3) with walls on every
    face, small enough that every path (interior, x/y wall bands, z walls,
    corners) is exercised;
  * the uniform-box kernel, when the stretched kernel is given uniform axes
    (its flux form reduces to the exact shift there);
  * conservation of the salinity to FP32 round-off.
"""
import numpy as np
import pytest

from ip_cu_lbm_b200.sim3d import Sim3D
from oracle.structured3d import W7, W19, Box3D
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def clustered(n, ratio=3.0):
    """Cells clustered toward the centreline, finest width 1, widest `ratio`."""
    xi = (np.arange(n) + 0.5) / n
    w = 1.0 + (ratio - 1.0) * np.abs(2.0 * xi - 1.0) ** 2
    w = w / w.min()
    return np.cumsum(w) - w / 2, w


def initial(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    S = 0.5 + 0.3 * np.sin(2 * np.pi * xx / nx) * np.cos(np.pi * zz / nz) * np.cos(np.pi * yy / ny)
    u = 1e-3 * np.sin(2 * np.pi * zz / nz)
    v = 1e-3 * np.cos(2 * np.pi * xx / nx)
    w = 1e-3 * np.sin(2 * np.pi * yy / ny)
    from oracle.structured3d import E19

    e = E19.astype(float)
    eu = e[:, 0, None, None, None] * u + e[:, 1, None, None, None] * v + e[:, 2, None, None, None] * w
    f = W19[:, None, None, None] * (3 * eu + 4.5 * eu ** 2 - 1.5 * (u * u + v * v + w * w))
    f = f + 1e-5 * W19[:, None, None, None] * rng.standard_normal(f.shape)
    g = W7[:, None, None, None] * S[None] * (1 + 4 * eu[:7])
    return f, g


PHYS = dict(tau=0.58, taus=0.53, g_bouss=1e-4, rho_sal=1e-3)


@pytest.mark.parametrize("ns", [3, 5])
def test_stretched_3d_matches_fp64_oracle(cuda, ns):
    nx, ny, nz = 44, 36, 12  # two CTA columns in x, five in y: interior, wall bands and tile seams
    X, WX = clustered(nx)
    Y, WY = clustered(ny)
    f, g = initial(nx, ny, nz, 3)
    b = Box3D(nx, ny, nz, x=X, wx=WX, y=Y, wy=WY, ns=ns, **PHYS)
    b.f, b.g = f.copy(), g.copy()
    s = Sim3D(nx, ny, nz, x=X, wx=WX, y=Y, wy=WY, ns=ns, **PHYS)
    s.set_state(f=f, g=g, F=np.zeros((3, nz, ny, nx)))
    for n in (1, 9):
        b.step(n)
        s.step(n)
    p, S, rho, u = b.moments()
    for name, mine, ref in (("ux", s.get("ux"), u[0]), ("uy", s.get("uy"), u[1]), ("uz", s.get("uz"), u[2]),
                            ("S", s.get("S"), S), ("p", s.get("p"), p)):
        err = rel_l2(mine, ref)
        assert err <= 1e-5, (ns, name, err)
    assert s.status() == 0
    s.close()


def test_stretched_kernel_on_uniform_axes_equals_uniform_kernel(cuda):
    nx, ny, nz = 40, 20, 10
    f, g = initial(nx, ny, nz, 5)
    a = Sim3D(nx, ny, nz, **PHYS)
    b = Sim3D(nx, ny, nz, x=np.arange(nx) + 0.5, wx=np.ones(nx), y=np.arange(ny) + 0.5, wy=np.ones(ny), ns=3,
              **PHYS)
    for s in (a, b):
        s.set_state(f=f, g=g, F=np.zeros((3, nz, ny, nx)))
        s.step(6)
        s.step_graph(8)
    for k in ("f", "g", "F"):
        err = rel_l2(b.get(k), a.get(k), floor=1e-30)
        assert err <= 1e-6, (k, err)
    a.close()
    b.close()


def test_stretched_salinity_conserved(cuda):
    nx, ny, nz = 48, 40, 24
    X, WX = clustered(nx)
    Y, WY = clustered(ny)
    f, g = initial(nx, ny, nz, 7)
    s = Sim3D(nx, ny, nz, x=X, wx=WX, y=Y, wy=WY, ns=3, **PHYS)
    s.set_state(f=f, g=g, F=np.zeros((3, nz, ny, nx)))
    area = WX[None, None, :] * WY[None, :, None]
    s0 = float((s.get("S") * area).sum())
    s.step_graph(200)
    s1 = float((s.get("S") * area).sum())
    assert abs(s1 - s0) <= 2e-6 * s0, (s0, s1)
    assert s.status() == 0
    s.close()
