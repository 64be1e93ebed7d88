"""The fused 3-D kernel (ipcu_sim3d_*, D3Q19 MRT + D3Q7 salinity, uniform
box, bounce-back) against the FP64 3-D oracle, rel-L2 <= 1e-5 in FP32; the
rest state; conservation; graph replay equal to direct steps."""
import numpy as np
import pytest

from ip_cu_lbm_b200.sim3d import Sim3D
from helpers import rel_l2
from oracle.structured3d import Box3D
from test_structured3d_oracle import _state

pytestmark = pytest.mark.gpu

PHYS = dict(tau=0.58, taus=0.53, g_bouss=1e-4, rho_sal=1e-3)


def _pair(nx, ny, nz, mrt, seed=1):
    b = Box3D(nx, ny, nz, mrt=mrt, **PHYS)
    b.f, b.g = _state(b, seed)
    s = Sim3D(nx, ny, nz, mrt=mrt, **PHYS)
    s.set_state(f=b.f, g=b.g, F=b.F)
    return b, s


@pytest.mark.parametrize("mrt", [True, False])
@pytest.mark.parametrize("dims", [(20, 12, 10), (33, 9, 17), (64, 16, 40)])
def test_fused3d_matches_oracle(cuda, mrt, dims):
    b, s = _pair(*dims, mrt)
    for n in (1, 25):
        b.step(n)
        s.step(n)
        p, S, rho, u = b.moments()
        for name, mine, ref in (("ux", s.get("ux"), u[0]), ("uy", s.get("uy"), u[1]), ("uz", s.get("uz"), u[2]),
                                ("S", s.get("S"), S), ("p", s.get("p"), p)):
            err = rel_l2(mine, ref, floor=1e-30)
            assert err <= 1e-5, (n, name, err)
    assert s.status() == 0


def test_rest_state_exact(cuda):
    s = Sim3D(20, 10, 8, g_bouss=0.0, rho_sal=0.0, s0=np.full(20 * 10 * 8, 0.4))
    s.step(30)
    assert not np.any(s.get("f"))
    assert np.all(np.abs(s.get("S") - 0.4) <= 2e-7)


def test_conservation(cuda):
    nx, ny, nz = 48, 24, 32
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    s0 = np.where(xx < nx // 2, 1.0, 0.0)
    s = Sim3D(nx, ny, nz, g_bouss=1e-4, rho_sal=1e-4, tau=0.55, taus=0.52, s0=s0)
    t0 = s.get("S").sum()
    s.step(300)
    assert abs(s.get("S").sum() - t0) <= 1e-4 * t0
    assert abs(s.get("p").sum()) <= 1e-5 * nx * ny * nz
    assert s.status() == 0


def test_graph_replay_equals_direct(cuda):
    b, s = _pair(40, 16, 24, True)
    _, r = _pair(40, 16, 24, True)
    s.step(21)
    r.step_graph(21)
    for k in ("ux", "uy", "uz", "S", "p"):
        assert np.array_equal(s.get(k), r.get(k)), k
