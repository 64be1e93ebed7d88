"""Generates tests/golden/reference_f32.npz: outputs of the reference's own
CUDA build (oracle/_ref/libipcu_ref.so, built from the reference sources by
oracle/Makefile) on small seeded inputs, one record per kernel of the
reference API plus LockExchange and moving-IBM step chains. Run on a GPU box:

    python tests/golden/make_golden.py [out.npz]

tests/test_oracle_golden.py checks the CPU oracle against these fixtures
without a GPU.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
ROOT = os.path.dirname(TESTS)
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)

from helpers import gpu_chain, mrt_mats, random_state  # noqa: E402
from ip_cu_lbm_b200 import cases  # noqa: E402
import test_ibm_gpu as tib  # noqa: E402
import test_legacy_gpu as tl  # noqa: E402

GOLDEN_CASES = {
    "q9": dict(Q=9, nx0=8, nz=6, divx=[1, 2, 4, 1, 1, 2, 1, 1], ratiox=4.0, dx=1.0, dt=1.0),
    "q27": dict(Q=27, nx0=3, ny0=3, nz=4, divx=[1, 2, 1], divy=[1, 2, 1], ratiox=2.0, ratioy=2.0, dx=1.0, dt=1.0),
}


def main(out):
    rec = {}
    saved_cases = dict(tl.CASES)
    tl.CASES.update(GOLDEN_CASES)
    for ck in GOLDEN_CASES:
        c, st = tl.make_inputs(ck, "f32")
        for k in ("items", "neib", "nextB", "nextK", "posx", "posy", "posz", "delX", "delY"):
            rec[f"{ck}/case/{k}"] = c[k]
        for a, wl in enumerate(c["walls"]):
            rec[f"{ck}/case/w{a + 1}"] = wl
        for k, v in st.items():
            rec[f"{ck}/in/{k}"] = v
        for i, (name, args, outs) in enumerate(tl.KERNELS):
            if "M" in args and "M" not in st:
                continue
            ref = tl.run_kernel("ref", name, args, c, st, "f32")
            for o in outs:
                rec[f"{ck}/k{i}/{o}"] = ref[o]
    tl.CASES.clear()
    tl.CASES.update(saved_cases)
    # LockExchange chain, 10 steps, bounce-back and slip
    c = cases.box_case(prec="f32", **GOLDEN_CASES["q9"])
    st = random_state(c, 31, tau=0.6, taus=0.55)
    for k, v in st.items():
        rec[f"le/in/{k}"] = v
    for slip in (0, 1):
        ref = gpu_chain(c, st, 10, "ref", slip=slip, mats=mrt_mats())
        for k in ("u", "w", "sal", "p", "f", "g", "rho"):
            rec[f"le/slip{slip}/{k}"] = getattr(ref, k)
    # moving-IBM chain, 5 steps
    c, body = cases.ibm_ellipse_case(nx0=24, nz=30, n_markers=16)
    st = random_state(c, 9, tau=0.7, taus=0.55, amp=1e-4)
    st.update(body)
    for k in ("uo", "vo", "wo"):
        st[k] = np.zeros(c["nt"], np.float32)
    st["sal"][:] = 0
    st["rho"][:] = 1000.0
    for k, v in st.items():
        rec[f"ibm/in/{k}"] = v
    ref = gpu_chain(c, st, 5, "ref", slip=1, kind="ibm", rhoH=1000.0)
    for k in ("posB", "velB", "angleVB", "quat", "posw", "Gw", "u", "w", "p", "lid", "f"):
        rec[f"ibm/out/{k}"] = getattr(ref, k)
    np.savez_compressed(out, **rec)
    print(f"wrote {out}: {len(rec)} arrays, {os.path.getsize(out) / 1e6:.2f} MB")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "reference_f32.npz"))
