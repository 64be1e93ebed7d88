"""The FP64 immersed-boundary oracle (oracle/ibm2d.py) on its own: the
Peskin kernel's moment conditions (the reference's weightFunction,
function/ibm.cu:61-66), rest state, symmetry, no-slip enforcement and a
stable settling at the density ratios near one where an explicit body
update of the marker reaction alone diverges."""
import numpy as np

from ip_cu_lbm_b200.cases import d2q9_mrt, ellipse_markers
from oracle.ibm2d import Body2D, IBBox, peskin4
from oracle.structured import Box


def make(rho_s=1.5, theta=0.0, grav=1e-4, xc=32.0, nx=64, nz=96):
    M, Minv, S = d2q9_mrt()
    b = Box(nx, nz, q_scalar=0, M=M, Minv=Minv, S=S, tau=0.56, rho_sal=0.0, g_bouss=0.0)
    X0, dS = ellipse_markers(8.0, 4.0, 48)
    body = Body2D(xc, 64.0, X0, dS, rho_s=rho_s, area=np.pi * 32, inertia_per_mass=20.0, theta=theta)
    body.a_b = (8.0, 4.0)
    return b, body, IBBox(b, body, rho_f=1.0, gravity=grav, iters=3)


def test_peskin4_moments():
    """Partition of unity, zero first moment and sum of squares 3/8 at any offset."""
    j = np.arange(-3, 4)
    for x in np.random.default_rng(1).uniform(0, 1, 32):
        ph = peskin4(x - j)
        assert abs(ph.sum() - 1) < 1e-14
        assert abs(((x - j) * ph).sum()) < 1e-14
        assert abs((ph ** 2).sum() - 0.375) < 1e-14
    assert peskin4(2.0) == 0.0 and peskin4(2.5) == 0.0


def test_ellipse_markers_equal_arc():
    X, dS = ellipse_markers(20.0, 10.0, 240)
    assert np.allclose((X[:, 0] / 20) ** 2 + (X[:, 1] / 10) ** 2, 1.0)
    seg = np.hypot(*np.diff(np.vstack([X, X[:1]]), axis=0).T)
    assert seg.std() / seg.mean() < 2e-3
    assert abs(dS.sum() - 96.88448) < 1e-3  # perimeter of the 20 x 10 ellipse


def test_rest_state_is_exact():
    b, body, ib = make(rho_s=1.0, grav=1e-3)
    ib.step(20)
    assert np.all(body.U == 0) and body.om == 0 and np.all(body.X == [32.0, 64.0])
    assert np.all(b.ux == 0) and np.all(b.uz == 0) and np.all(b.fext == 0)


def test_symmetric_body_sinks_straight():
    b, body, ib = make(rho_s=1.5, theta=0.0)
    ib.step(60)
    assert body.U[1] < 0 and body.X[1] < 64.0
    assert abs(body.X[0] - 32.0) < 1e-12 and abs(body.om) < 1e-15


def test_mdf_enforces_no_slip():
    b, body, ib = make(rho_s=1.5, theta=0.3)
    ib.step(60)
    X, Ub = body.markers()
    K, I, W = ib._stencil(X)
    Us = np.stack([(W * b.ux[K, I]).sum(1), (W * b.uz[K, I]).sum(1)], 1)
    assert np.abs(Us - Ub).max() < 0.05 * np.abs(Ub).max()


def test_settling_stable_near_unit_density_ratio():
    for rho_s in (1.1, 1.5):
        b, body, ib = make(rho_s=rho_s, theta=np.pi / 4)
        ib.step(300)
        assert np.isfinite(body.U).all() and abs(body.th - np.pi / 4) < 0.05
        assert -0.01 < body.U[1] < 0  # sinking, well below the lattice speed
        assert np.abs(b.uz).max() < 0.01


def test_body_list_of_one_equals_single_body():
    """IBBox over a list of bodies reduces to the one-body step."""
    M, Minv, S = d2q9_mrt()
    X0, dS = ellipse_markers(6.0, 3.0, 32)
    runs = []
    for as_list in (False, True):
        b = Box(40, 48, M=M, Minv=Minv, S=S, q_scalar=0, tau=0.56, rho_sal=0.0, g_bouss=0.0)
        bd = Body2D(20.0, 30.0, X0, dS, rho_s=1.5, area=np.pi * 18.0, inertia_per_mass=45.0 / 4, theta=0.3)
        bd.a_b = (6.0, 3.0)
        IBBox(b, [bd] if as_list else bd, rho_f=1.0, gravity=1e-4, iters=3).step(5)
        runs.append((b.ux.copy(), b.uz.copy(), np.array([*bd.X, *bd.U, bd.th, bd.om])))
    for x, y in zip(*runs):
        assert np.array_equal(x, y)
