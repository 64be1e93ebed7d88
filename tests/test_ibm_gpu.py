"""Immersed-boundary entries of libipcu vs the reference's own CUDA build on
the settling-ellipse set-up (ref: EllipticalFall2/EllipticalFallxz.cu), kernel
by kernel and as the moving-body step chain (ibm_step order)."""
import numpy as np
import pytest

from ip_cu_lbm_b200 import cases
from helpers import gpu_chain, random_state, rel_l2

pytestmark = pytest.mark.gpu


def _ref_ok():
    from oracle import oracle as _o

    return _o.ref_available()


def ibm_inputs(seed=3, n_markers=24):
    c, body = cases.ibm_ellipse_case(n_markers=n_markers)
    st = random_state(c, seed, tau=0.7, taus=0.55, amp=1e-3)
    dt = c["dtype"]
    rng = np.random.default_rng(seed)
    st.update(body)
    nt = c["nt"]
    st["Fx"], st["Fy"], st["Fz"] = (1e-3 * rng.standard_normal(nt)).astype(dt), np.zeros(nt, dt), (
        1e-3 * rng.standard_normal(nt)).astype(dt)
    st["velw"] = (1e-3 * rng.standard_normal(3 * n_markers)).astype(dt)
    st["Gw"] = (1e-3 * rng.standard_normal(3 * n_markers)).astype(dt)
    st["FB"] = np.array([1e-3, 0, -2e-3], dt)
    st["Torque"] = np.array([0, 1e-6, 0], dt)
    st["angleVB"] = np.array([0, 0.1, 0], dt)
    st["velB"] = np.array([1e-3, 0, -1e-3], dt)
    for k in ("uo", "vo", "wo"):
        st[k] = np.zeros(nt, dt)
    return c, st


IB_KERNELS = [
    ("get_IBMGw2", ["items", "lid", "neib", "f", "tau", "posx", "posy", "posz", "posw", "posB", "nB", "u", "v", "w",
                    "velw", "Fx", "Fy", "Fz", "Gw", 1000.0], ["Fx", "Fy", "Fz", "Gw"]),
    ("update_velIBM", ["items", "lid", "f", "ftmp", "p", "tau", "u", "v", "w", "uo", "vo", "wo", "Fx", "Fy", "Fz"],
     ["f", "p", "u", "v", "w"]),
    ("update_IBbody", ["items", 0, "massB", "densB", "inertia", "FB", "posB", "Torque", "velB", "quat", "quaS",
                       "angleVB", "posw", "Gw", "quatold", 1000.0],
     ["FB", "posB", "Torque", "velB", "quat", "quaS", "angleVB", "quatold"]),
    ("update_IBpoint", ["items", 0, "posB", "velB", "angleVB", "quaS", "posw", "oposw", "nB", "onB", "velw"],
     ["posw", "nB", "velw"]),
    ("search_IBlattice", ["items", 0, "lid", "neib", "posx", "posy", "posz", "posw"], ["lid"]),
    ("IB_directForcing", ["items", "lid", "neib", "posx", "posy", "posz", "posw", "u", "v", "w", "velw", "Fx", "Fy",
                          "Fz", "Gw"], ["Fx", "Fy", "Fz", "Gw"]),
    ("SPM", ["items", 0.004, "posB", "f", "ftmp", "tau", "posx", "posz", "Fx", "Fy", "Fz", "u", "v", "w", "velw"],
     ["f", "ftmp", "Fx", "Fy", "Fz"]),
    ("SPM_ellipse", ["items", 0.005, 0.0025, "quaS", "posB", "f", "tau", "posx", "posy", "posz", "u", "v", "w",
                     "velB", "angleVB"], ["f"]),
]


def run(backend, name, args, c, st):
    import torch

    from ip_cu_lbm_b200 import _lib

    dev = torch.device("cuda:0")
    host = dict(st)
    for k in ("items", "neib", "posx", "posy", "posz", "delX", "delY"):
        host[k] = c[k]
    host["ftmp"] = st["f"].copy()
    bufs = {k: torch.as_tensor(np.ascontiguousarray(v), device=dev,
                               dtype=torch.float32 if np.asarray(v).dtype.kind == "f" else torch.int32).clone()
            for k, v in host.items()}
    res = [bufs[a] if isinstance(a, str) else a for a in args]
    nt = c["nt"]
    if backend == "ref":
        from oracle import oracle as _o

        assert _o.ref()(name, "f32", *res, n=nt) == 0
    else:
        _lib.check(_lib.legacy()(name, "f32", *res, tail=(nt, torch.cuda.current_stream(dev).cuda_stream)), name)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in bufs.items()}


@pytest.mark.parametrize("idx", range(len(IB_KERNELS)))
def test_ibm_kernel_matches_reference(cuda, idx):
    if not _ref_ok():
        pytest.skip("reference build (oracle/_ref) not present")
    name, args, outs = IB_KERNELS[idx]
    c, st = ibm_inputs()
    mine = run("ipcu", name, args, c, st)
    ref = run("ref", name, args, c, st)
    for o in outs:
        if o == "lid":
            assert np.array_equal(mine[o], ref[o])
            continue
        err = rel_l2(mine[o], ref[o], floor=1e-30)
        assert err <= 2e-6, (name, o, err)


@pytest.mark.parametrize("nsteps", [1, 5, 25])
def test_ibm_chain_matches_reference(cuda, nsteps):
    if not _ref_ok():
        pytest.skip("reference build (oracle/_ref) not present")
    c, body = cases.ibm_ellipse_case(n_markers=24)
    st = random_state(c, 9, tau=0.7, taus=0.55, amp=1e-4)
    st.update(body)
    nt, dt = c["nt"], c["dtype"]
    for k in ("uo", "vo", "wo"):
        st[k] = np.zeros(nt, dt)
    st["sal"][:] = 0
    st["rho"][:] = 1000.0
    mine = gpu_chain(c, st, nsteps, "ipcu", slip=1, kind="ibm", rhoH=1000.0)
    ref = gpu_chain(c, st, nsteps, "ref", slip=1, kind="ibm", rhoH=1000.0)
    for k in ("posB", "velB", "angleVB", "quat", "posw", "Gw", "u", "w", "p"):
        err = rel_l2(getattr(mine, k), getattr(ref, k), floor=1e-30)
        assert err <= 1e-5, (k, err)
    assert np.array_equal(mine.lid, ref.lid)
