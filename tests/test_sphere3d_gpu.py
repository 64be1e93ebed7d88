"""The moving sphere on the 3-D solver (ipcu_sim3d_ib_attach: multi-direct
forcing with the Peskin-4 kernel per axis, FP64 body update) against the
FP64 oracle (oracle/ibm3d.py on oracle/structured3d.py) on a uniform box and
on stretched x and y axes; the rest state; graph replay equal to direct
steps; snapshots refused with a sphere."""
import numpy as np
import pytest

from ip_cu_lbm_b200.sim3d import Sim3D
from oracle.ibm3d import IBBox3D, Sphere3D
from oracle.structured3d import Box3D
from helpers import rel_l2

pytestmark = pytest.mark.gpu

NX, NY, NZ = 24, 24, 36
R, NM = 4.0, 200
PHYS = dict(tau=0.56, taus=0.52, rho_sal=0.0, g_bouss=0.0)


def axes(stretched):
    if not stretched:
        return {}
    def ax(n, ratio=1.6):
        xi = (np.arange(n) + 0.5) / n
        w = 1.0 + (ratio - 1.0) * np.abs(2.0 * xi - 1.0) ** 2
        w = w / w.min()
        return np.cumsum(w) - w / 2, w
    x, wx = ax(NX)
    y, wy = ax(NY)
    return dict(x=x, wx=wx, y=y, wy=wy, ns=3)


def centre(kw):
    x = kw.get("x", np.arange(NX) + 0.5)
    y = kw.get("y", np.arange(NY) + 0.5)
    return 0.5 * (x[NX // 2 - 1] + x[NX // 2]), 0.5 * (y[NY // 2 - 1] + y[NY // 2])


def run_pair(steps, stretched=False, rho_s=1.5, grav=1e-4):
    kw = axes(stretched)
    xc, yc = centre(kw)
    zc = 22.0
    s = Sim3D(NX, NY, NZ, **PHYS, **kw)
    s.attach_sphere(xc, yc, zc, R, markers=NM, rho_s=rho_s, gravity=grav)
    s.step(steps)
    b = Box3D(NX, NY, NZ, **PHYS, **kw)
    sp = Sphere3D(xc, yc, zc, R, NM, rho_s=rho_s)
    IBBox3D(b, sp, rho_f=1.0, gravity=grav).step(steps)
    return s, b, sp, (xc, yc, zc)


@pytest.mark.parametrize("stretched", [False, True])
def test_sphere_matches_fp64_oracle(cuda, stretched):
    steps = 60
    s, b, sp, X0 = run_pair(steps, stretched)
    assert s.status() == 0
    d = s.body()
    moved = np.abs(sp.X - np.array(X0)).max()
    dpos = np.abs(d["X"] - sp.X).max() / moved
    dvel = np.abs(d["U"] - sp.U).max() / np.abs(sp.U).max()
    print(f"sphere ({'stretched' if stretched else 'uniform'}): w {d['U'][2]:.6e} vs FP64 {sp.U[2]:.6e}; "
          f"position rel {dpos:.2e}, velocity rel {dvel:.2e}")
    assert sp.U[2] < 0  # it sinks
    assert dpos < 1e-4 and dvel < 1e-4, (dpos, dvel)
    p, S, rho, u = b.moments()
    for name, ref in (("ux", u[0]), ("uy", u[1]), ("uz", u[2])):
        e = rel_l2(s.get(name), ref)
        assert e < 1e-4, (name, e)
    s.close()


def test_neutral_sphere_stays_at_rest(cuda):
    s = Sim3D(NX, NY, NZ, **PHYS)
    s.attach_sphere(12.0, 12.0, 18.0, R, markers=NM, rho_s=1.0, gravity=1e-3)
    s.step(20)
    d = s.body()
    assert np.all(d["U"] == 0.0) and np.all(d["omega"] == 0.0)
    assert np.all(d["X"] == np.array([12.0, 12.0, 18.0]))
    assert np.all(s.get("uz") == 0.0)
    s.close()


def test_graph_replay_equals_direct_steps(cuda, tmp_path):
    """The update's sums run in a fixed order (pairs listed per cell and
    sorted): graph replay and direct steps agree bit for bit."""
    a = Sim3D(NX, NY, NZ, **PHYS)
    b = Sim3D(NX, NY, NZ, **PHYS)
    for s in (a, b):
        s.attach_sphere(12.3, 11.8, 22.0, R, markers=NM, rho_s=1.5, gravity=1e-4)
    a.step(30)
    b.step_graph(30)
    da, db = a.body(), b.body()
    for k in da:
        assert np.array_equal(da[k], db[k]), k
    assert np.array_equal(a.get("f"), b.get("f"))
    with pytest.raises(Exception):
        a.save(tmp_path / "s.ipcu3")  # the sphere's state is not part of the 3-D snapshot
    a.close()
    b.close()
