"""Device geometry set-up (ipcu_build_box_device_*, ipcu_nearest_cells_*)
against the host builders and the oracle's restatement of the case drivers'
nearest-cell search (ref: LockExchange/LockExchange.cu:55-127,
function/basic.cu:203-237, SphereFallSuzuki2018/SphereSuzuki.cu:268-275)."""
import numpy as np
import pytest

from oracle.oracle import oracle


def _np_nearest(px, py, pz, posw):
    """numpy statement of the same search: float32 differences, squares in
    double, sqrt rounded to float32, first index among equal minima."""
    out = []
    for m in posw.reshape(-1, 3):
        d = ((px - m[0]).astype(np.float64) ** 2 + (py - m[1]).astype(np.float64) ** 2
             + (pz - m[2]).astype(np.float64) ** 2)
        out.append(int(np.argmin(np.sqrt(d).astype(np.float32))))
    return np.array(out, np.int32)


def _oracle_nearest(px, py, pz, nc, posw):
    return oracle().nearest_cells(px, py, pz, nc, posw)


def _markers(rng, n, lo, hi):
    return rng.uniform(lo, hi, (n, 3)).astype(np.float32)


def test_oracle_nearest_matches_numpy_statement():
    from ip_cu_lbm_b200.cases import box_case

    case = box_case(Q=9, nx0=12, nz=10, divx=[1] * 4 + [2] * 4 + [1] * 4, dx=1e-2, ratiox=2.0)
    rng = np.random.default_rng(3)
    nc = case["nc"]
    px, py, pz = (case[k][:nc].copy() for k in ("posx", "posy", "posz"))
    posw = _markers(rng, 40, [0, 0, 0], [px.max(), 0, pz.max()])
    posw[:, 1] = py[0]
    # a marker exactly between two cells of a row: both at the same distance
    posw[0] = [(px[0] + px[case["nz"]]) / 2, py[0], pz[0]]
    got = _oracle_nearest(px, py, pz, nc, posw.ravel().copy())
    np.testing.assert_array_equal(got, _np_nearest(px, py, pz, posw))
    assert got[0] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("Q,nx0,ny0,nz,divx,divy,ratiox,ratioy", [
    (9, 12, 1, 10, [1] * 4 + [2] * 4 + [4] * 4, [1], 4.0, 1.0),
    (9, 40, 1, 33, None, None, 1.0, 1.0),
    (27, 5, 4, 6, [1, 2, 1, 2, 1], [2, 1, 1, 2], 2.0, 2.0),
])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_device_box_matches_host(cuda, Q, nx0, ny0, nz, divx, divy, ratiox, ratioy, prec):
    from ip_cu_lbm_b200.cases import box_case, box_grid_device

    kw = dict(Q=Q, nx0=nx0, ny0=ny0, nz=nz, divx=divx, divy=divy, dx=1e-2, ratiox=ratiox, ratioy=ratioy, prec=prec)
    h = box_case(**kw)
    d = box_grid_device(**kw)
    assert (d["nc"], d["nw"], d["nt"]) == (h["nc"], h["nw"], h["nt"])
    np.testing.assert_array_equal(d["lnum"].cpu().numpy(), h["lnum"])
    np.testing.assert_array_equal(d["neib"].cpu().numpy(), h["neib"])
    np.testing.assert_array_equal(d["owner"].cpu().numpy(), h["owner"])
    for k in ("posx", "posy", "posz", "delX", "delY"):
        np.testing.assert_array_equal(d[k].cpu().numpy(), h[k], err_msg=k)


@pytest.mark.gpu
def test_device_box_capacity_error(cuda):
    import ctypes

    import torch

    from ip_cu_lbm_b200 import _lib

    L = _lib.lib()
    divx = np.ones(8, np.int32)
    divy = np.ones(1, np.int32)
    cap = 8 * 8  # room for the fluid cells only, none for the ghosts
    t = [torch.empty(cap * 9, dtype=torch.int32, device=cuda) for _ in range(3)]
    g = [torch.empty(cap, dtype=torch.float32, device=cuda) for _ in range(5)]
    nc, nw = ctypes.c_int64(), ctypes.c_int64()
    st = L.ipcu_build_box_device_f32(9, 8, 1, 8, 1.0, 1.0, 1.0, divx.ctypes.data, divy.ctypes.data,
                                     t[0].data_ptr(), t[1].data_ptr(), *[x.data_ptr() for x in g], cap,
                                     t[2].data_ptr(), ctypes.byref(nc), ctypes.byref(nw), None)
    assert st == -4  # IPCU_ERR_CAPACITY
    st = L.ipcu_build_box_device_f32(8, 8, 1, 8, 1.0, 1.0, 1.0, divx.ctypes.data, divy.ctypes.data,
                                     t[0].data_ptr(), t[1].data_ptr(), *[x.data_ptr() for x in g], cap,
                                     t[2].data_ptr(), ctypes.byref(nc), ctypes.byref(nw), None)
    assert st < 0  # Q must be 9 or 27


@pytest.mark.gpu
@pytest.mark.parametrize("nx0,nz,nm", [(12, 10, 37), (256, 128, 300)])
def test_nearest_cells_match_oracle(cuda, nx0, nz, nm):
    import torch

    from ip_cu_lbm_b200.cases import box_case, nearest_cells

    divx = [1] * (nx0 // 3) + [2] * (nx0 // 3) + [1] * (nx0 - 2 * (nx0 // 3))
    case = box_case(Q=9, nx0=nx0, nz=nz, divx=divx, dx=1e-2, ratiox=2.0)
    nc = case["nc"]
    rng = np.random.default_rng(nx0)
    px, py, pz = (case[k][:nc].copy() for k in ("posx", "posy", "posz"))
    posw = _markers(rng, nm, [0, 0, 0], [px.max() * 1.05, 0, pz.max() * 1.05])
    posw[:, 1] = py[0]
    posw[0] = [(px[0] + px[nz]) / 2, py[0], pz[0]]                  # tie in x
    posw[1] = [px[5 * nz + 3], py[0], (pz[3] + pz[4]) / 2]            # tie in z
    want = _oracle_nearest(px, py, pz, nc, posw.ravel().copy())
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    # ghosts (indices >= nc) must never be chosen: pass the full arrays
    got = nearest_cells(dev(case["posx"]), dev(case["posy"]), dev(case["posz"]), nc, dev(posw))
    np.testing.assert_array_equal(got.cpu().numpy(), want)
