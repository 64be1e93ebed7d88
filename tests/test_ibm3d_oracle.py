"""The FP64 3-D immersed-boundary oracle (oracle/ibm3d.py) on its own: the
Fibonacci markers cover the sphere's area, the index-space Peskin weights
form a partition of unity on a stretched axis and spread a marker force
without loss, a neutrally buoyant sphere in fluid at rest stays at rest, and
a heavy one sinks without drifting sideways."""
import numpy as np

from oracle.ibm2d import peskin4
from oracle.ibm3d import IBBox3D, Sphere3D, index_coord, sphere_markers
from oracle.structured3d import Box3D


def test_markers_cover_the_sphere():
    r, dA = sphere_markers(3.0, 400)
    assert np.allclose(np.linalg.norm(r, axis=1), 3.0)
    assert abs(dA.sum() - 4 * np.pi * 9.0) < 1e-9
    assert np.abs(r.mean(0)).max() < 0.02  # nearly balanced about the centre


def test_index_space_weights_partition_of_unity():
    w = 1.0 + 0.6 * np.abs(np.linspace(-1, 1, 30)) ** 2
    xc = np.cumsum(w) - w / 2
    for x in np.linspace(xc[3], xc[-4], 17):
        s = index_coord(xc, np.array([x]))[0]
        i0 = int(np.floor(s)) - 1
        W = peskin4(np.arange(i0, i0 + 4) - s)
        assert abs(W.sum() - 1.0) < 1e-12
        assert abs((W * (np.arange(i0, i0 + 4) - s)).sum()) < 1e-12  # zero first moment


def _box():
    return Box3D(20, 20, 28, tau=0.56, taus=0.52, rho_sal=0.0, g_bouss=0.0)


def test_neutral_sphere_at_rest():
    b = _box()
    sp = Sphere3D(10.0, 10.0, 16.0, 3.0, 120, rho_s=1.0)
    IBBox3D(b, sp, rho_f=1.0, gravity=1e-3).step(4)
    assert np.all(sp.U == 0.0) and np.all(b.f == 0.0)


def test_heavy_sphere_sinks_straight():
    b = _box()
    sp = Sphere3D(10.0, 10.0, 16.0, 3.0, 120, rho_s=1.5)
    IBBox3D(b, sp, rho_f=1.0, gravity=1e-4).step(12)
    assert sp.U[2] < 0
    assert np.abs(sp.U[:2]).max() < 1e-3 * abs(sp.U[2])
