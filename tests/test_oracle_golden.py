"""The CPU oracle against golden outputs of the reference's own CUDA build
(tests/golden/reference_f32.npz, made by tests/golden/make_golden.py on a
GPU box from the unmodified reference sources). Runs without a GPU.

Per kernel: FP32 oracle within 2e-6 rel-L2 of the reference (same float
formulas; FMA contraction and atomic order differ), FP64 oracle within 1e-5.
Step chains (10 LockExchange steps, 5 moving-IBM steps): FP32 oracle within
1e-5, FP64 oracle within 1e-4 (chains amplify the FP32 rounding of the
reference)."""
import os
from types import SimpleNamespace

import numpy as np
import pytest

from helpers import oracle_chain, rel_l2, mrt_mats
import test_legacy_gpu as tl

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_f32.npz")
pytestmark = pytest.mark.skipif(not os.path.exists(GOLDEN), reason="golden fixtures not generated yet")


def _load():
    d = np.load(GOLDEN)
    return {k: d[k] for k in d.files}


G = _load() if os.path.exists(GOLDEN) else {}


def _case(ck):
    c = {k.split("/")[-1]: v for k, v in G.items() if k.startswith(f"{ck}/case/")}
    it = c["items"]
    c["Q"], c["nc"], c["nw"] = int(it[6]), int(it[10]), int(it[11])
    c["nt"] = c["nc"] + c["nw"]
    c["walls"] = [c.pop(f"w{a + 1}") for a in range(6)]
    c["dtype"] = np.float32
    return c


def _inputs(prefix):
    return {k[len(prefix):]: v for k, v in G.items() if k.startswith(prefix)}


@pytest.mark.parametrize("ck", ["q9", "q27"])
@pytest.mark.parametrize("idx", range(len(tl.KERNELS)))
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_oracle_kernel_matches_reference(ck, idx, prec):
    name, args, outs = tl.KERNELS[idx]
    if f"{ck}/k{idx}/{outs[0]}" not in G:
        pytest.skip("no fixture for this kernel/case")
    c = _case(ck)
    st = _inputs(f"{ck}/in/")
    got = tl.run_kernel("oracle", name, args, c, st, prec)
    tol = 2e-6 if prec == "f32" else 1e-5
    for o in outs:
        ref = G[f"{ck}/k{idx}/{o}"]
        err = rel_l2(got[o], ref, floor=1e-30)
        assert err <= tol, (name, o, err)


def _le_case(prec):
    from ip_cu_lbm_b200 import cases

    c = cases.box_case(prec=prec, Q=9, nx0=8, nz=6, divx=[1, 2, 4, 1, 1, 2, 1, 1], ratiox=4.0, dx=1.0, dt=1.0)
    # the fixture was made on the grid this build produces (host set-up is bit-exact)
    assert np.array_equal(c["neib"], G["q9/case/neib"])
    return c


@pytest.mark.parametrize("slip", [0, 1])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_oracle_lockexchange_chain(slip, prec):
    c = _le_case(prec)
    st = {k: v.astype(c["dtype"]) if v.dtype.kind == "f" else v for k, v in _inputs("le/in/").items()}
    out = oracle_chain(c, st, 10, slip=slip, mats=mrt_mats())
    nc = c["nc"]
    tol = 1e-5 if prec == "f32" else 1e-4
    for k in ("u", "w", "sal", "p"):
        err = rel_l2(getattr(out, k)[:nc], G[f"le/slip{slip}/{k}"][:nc], floor=1e-30)
        assert err <= tol, (k, err)


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_oracle_ibm_chain(prec):
    from ip_cu_lbm_b200 import cases

    c, _ = cases.ibm_ellipse_case(nx0=24, nz=30, n_markers=16, prec=prec)
    st = {k: v.astype(c["dtype"]) if v.dtype.kind == "f" else v for k, v in _inputs("ibm/in/").items()}
    out = oracle_chain(c, st, 5, slip=1, kind="ibm", rhoH=1000.0)
    tol = 1e-5 if prec == "f32" else 1e-4
    for k in ("posB", "velB", "angleVB", "quat", "posw", "Gw", "u", "w", "p"):
        err = rel_l2(getattr(out, k), G[f"ibm/out/{k}"], floor=1e-30)
        assert err <= tol, (k, err)
    assert np.array_equal(out.lid, G["ibm/out/lid"])
