"""Host set-up helpers (ghost cells, wall lists, slip tables, lattice
constants, MRT matrices): structural invariants, and bit-exact agreement
with the reference's own host functions where the reference build
(oracle/_ref) is present. Integer work must match exactly."""
import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT
from ip_cu_lbm_b200 import cases

HAVE_REF = os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libipcu_ref.so"))
needs_ref = pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")

CASES = [
    dict(Q=9, nx0=7, nz=5),
    dict(Q=9, nx0=6, nz=4, divx=[1, 2, 4, 2, 1, 1]),
    dict(Q=9, nx0=1, nz=3),
    dict(Q=27, nx0=4, ny0=3, nz=5, divx=[1, 2, 2, 1], divy=[1, 2, 1]),
    dict(Q=27, nx0=3, ny0=3, nz=3),
]


@pytest.mark.parametrize("kw", CASES)
def test_ghost_structure(kw):
    c = cases.box_case(**kw)
    Q, nc, nw, nb = c["Q"], c["nc"], c["nw"], c["neib"].reshape(-1, c["Q"])
    kinv = {9: [0, 3, 4, 1, 2, 7, 8, 5, 6],
            27: [0, 3, 4, 1, 2, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15, 26, 25, 24, 23, 22, 21, 20, 19]}[Q]
    assert (nb[:nc] >= 0).all() and (nb < nc + nw).all()
    for g in range(nc, nc + nw):
        o = nb[g, 0]
        assert o == c["owner"][g - nc] and o < nc
        for k in range(1, Q):
            if nb[o, k] == g:
                assert nb[g, kinv[k]] == o
            elif nb[g, k] != o:
                assert nb[g, k] == g
    # every fluid cell with a missing neighbour owns exactly one ghost
    open_cells = [i for i in range(nc) if (nb[i, 1:] >= nc).any()]
    assert sorted(open_cells) == sorted(c["owner"].tolist())


def _ref_lib():
    from oracle import oracle as _o

    return _o.ref()


@needs_ref
@pytest.mark.parametrize("kw", CASES)
def test_set_neibghor_wall_matches_reference(kw):
    c = cases.box_case(**kw)
    R = _ref_lib().lib
    Q, nc = c["Q"], c["nc"]
    NX, NY, nz = c["NX"], c["NY"], c["nz"]
    # rebuild the pre-ghost neighbour table with -1 holes
    nb = c["neib"].reshape(-1, Q)[:nc].copy()
    nb[nb >= nc] = -1
    cell_in = [np.ascontiguousarray(c[k][:nc], np.float32) for k in
               ("posx", "posx", "posx", "posx", "posy", "posz", "delX", "delY", "posx", "posx", "posx")]
    q_in = [np.zeros(nc * Q, np.float32) for _ in range(3)]
    cap = 2 * nc + 8
    neib_out = np.zeros(cap * Q, np.int32)
    cell_out = [np.zeros(cap, np.float32) for _ in range(11)]
    q_out = [np.zeros(cap * Q, np.float32) for _ in range(3)]
    CP = ctypes.c_void_p
    divx = np.zeros(NX, np.int32)
    divy = np.zeros(NY, np.int32)
    nt = R.ref_set_neibghor_wall_f32(NX, NY, nz, Q, nc, c["lnum"].ctypes.data, divx.ctypes.data, divy.ctypes.data,
                                     np.ascontiguousarray(nb.ravel()).ctypes.data,
                                     (CP * 11)(*[a.ctypes.data for a in cell_in]),
                                     (CP * 3)(*[a.ctypes.data for a in q_in]), cap, neib_out.ctypes.data,
                                     (CP * 11)(*[a.ctypes.data for a in cell_out]),
                                     (CP * 3)(*[a.ctypes.data for a in q_out]))
    assert nt == c["nt"]
    np.testing.assert_array_equal(neib_out[: nt * Q], c["neib"])
    # ghosts carry their owner's geometry
    np.testing.assert_array_equal(cell_out[5][:nt], c["posz"])
    np.testing.assert_array_equal(cell_out[6][:nt], c["delX"])


@needs_ref
@pytest.mark.parametrize("kw", CASES)
def test_walls_and_slip_tables_match_reference(kw):
    c = cases.box_case(**kw)
    R = _ref_lib().lib
    Q, nc, nw = c["Q"], c["nc"], c["nw"]
    it = c["items"]
    walls = [np.zeros(max(nc, 1), np.int32) for _ in range(6)]
    sizes = np.zeros(6, np.int32)
    rc = R.ref_set_walln_f32(it.ctypes.data, len(it), c["neib"].ctypes.data, len(c["neib"]), nc,
                             (ctypes.c_void_p * 6)(*[w.ctypes.data for w in walls]), sizes.ctypes.data)
    assert rc == 0
    for a in range(6):
        np.testing.assert_array_equal(walls[a][: sizes[a]], c["walls"][a])
    nK = np.zeros(nw * Q, np.int32)
    nB = np.zeros(nw * Q, np.int32)
    n = R.ref_set_bound_f32(2 if Q == 9 else 3, it.ctypes.data, len(it), nc, c["neib"].ctypes.data,
                            len(c["neib"]), nK.ctypes.data, nB.ctypes.data)
    assert n == nw * Q
    np.testing.assert_array_equal(nK, c["nextK"][: nw * Q])
    np.testing.assert_array_equal(nB, c["nextB"][: nw * Q])


@needs_ref
@pytest.mark.parametrize("Q,dx,dt", [(9, 0.001, 0.001), (27, 0.001, 0.00025), (9, 1.0, 1.0)])
def test_setc_matches_reference(Q, dx, dt):
    R = _ref_lib().lib
    out = [ctypes.c_double() for _ in range(3)]
    arrs = [np.zeros(27) for _ in range(4)]
    R.ref_setc(Q, dx, dt, 9, *[ctypes.byref(o) for o in out], *[a.ctypes.data for a in arrs])
    c, tau, taus, cx, cy, cz, w = cases.setc(Q, dx, dt)
    assert (c, tau, taus) == tuple(o.value for o in out)
    for mine, ref in zip((cx, cy, cz, w), arrs):
        np.testing.assert_array_equal(mine, ref[:Q])


@needs_ref
@pytest.mark.parametrize("Q", [9, 27])
def test_mrt_matrices_match_reference(Q):
    from oracle import oracle as _o

    R = _ref_lib().lib
    M, S, Mi, MM = np.zeros((Q, Q)), np.zeros(Q), np.zeros((Q, Q)), np.zeros((Q, Q))
    assert R.ref_set_M_f64(_o.REF_INPUT_DIR.encode(), Q, M.ctypes.data, S.ctypes.data, Mi.ctypes.data,
                           MM.ctypes.data) == 0
    from ip_cu_lbm_b200 import _lib

    Min, Sin, Miin = np.zeros((Q, Q)), np.zeros(Q), np.zeros((Q, Q))
    _lib.check(_lib.lib().ipcu_read_M_csv(_o.REF_INPUT_DIR.encode(), Q, Min.ctypes.data, Sin.ctypes.data,
                                          Miin.ctypes.data))
    M2, S2, Mi2, MM2 = cases.set_M(Q, Min, Sin, Miin)
    np.testing.assert_array_equal(M2, M)
    np.testing.assert_array_equal(S2, S)
    np.testing.assert_allclose(MM2, MM, rtol=0, atol=1e-15)
    if Q == 9:
        # the built-in Lallemand-Luo basis is the reference's input matrix
        Mb, Mib, Sb = cases.d2q9_mrt()
        np.testing.assert_array_equal(Mb, M)
        np.testing.assert_allclose(Mib, Mi, atol=1e-15)
        np.testing.assert_array_equal(Sb, Sin)
