"""Reference-compatible kernel entries of libipcu vs the reference's own CUDA
build (oracle/_ref) and vs the CPU oracle, kernel by kernel and as the
LockExchange step chain, on identical inputs.

Tolerances (FP32 path): per-kernel relative L2 <= 2e-6 against the reference
build (same float semantics, FMA contraction and summation order may differ),
<= 1e-5 after chains of steps; FP64 entries vs the FP64 oracle <= 1e-12."""
import numpy as np
import pytest

from ip_cu_lbm_b200 import cases
from helpers import gpu_chain, mrt_mats, oracle_chain, random_state, rel_l2

pytestmark = pytest.mark.gpu

CASES = {
    "q9": dict(Q=9, nx0=10, nz=7, divx=[1, 1, 2, 4, 1, 1, 2, 1, 1, 1], ratiox=4.0, dx=1.0, dt=1.0),
    "q9u": dict(Q=9, nx0=12, nz=6, dx=1.0, dt=1.0),
    "q27": dict(Q=27, nx0=5, ny0=4, nz=5, divx=[1, 2, 4, 1, 1], divy=[1, 2, 1, 1], ratiox=4.0, ratioy=2.0,
                dx=1.0, dt=1.0),
}

# name, arguments (buffer keys or literal scalars), outputs
KERNELS = [
    ("equ_f", ["items", "feq", "p", "u", "v", "w"], ["feq"]),
    ("equ_g", ["items", "feq", "sal", "u", "v", "w"], ["feq"]),
    ("Force", ["items", 1, "neib", "f", "feq", "tau", "Fk", "Fx", "Fy", "Fz", "p", "rho", "sal", "phi", "u", "v",
               "w", "delX", "delY", "posx", "posy", "posz"], ["Fk", "Fx", "Fy", "Fz"]),
    ("Force", ["items", 0, "neib", "f", "feq", "tau", "Fk", "Fx", "Fy", "Fz", "p", "rho", "sal", "phi", "u", "v",
               "w", "delX", "delY", "posx", "posy", "posz"], ["Fk", "Fx", "Fy", "Fz"]),
    ("col_f_MRT", ["items", "tau", "f", "ftmp", "feq", "Fk", "M", "Minv", "S", "MM"], ["f", "ftmp", "feq"]),
    ("col_f_SRT", ["items", "tau", "f", "ftmp", "feq", "Fk"], ["f", "ftmp", "feq"]),
    ("col_g_reg", ["items", "taus", "g", "ftmp", "feq", "sal", "u", "v", "w"], ["g", "ftmp", "feq"]),
    ("col_PF", ["items", "neib", "taus", "g", "ftmp", "feq", "phi", "u", "v", "w", "phio", "uo", "vo", "wo", "posx",
                "posy", "posz"], ["g", "ftmp", "feq", "phio", "uo", "vo", "wo"]),
    ("update_scalar", ["items", "g", "sal"], ["sal"]),
    ("update_rho", ["items", 1.0, 1000.0, "f", "Fx", "Fy", "Fz", "p", "sal", "phi", "rho", "u", "v", "w"],
     ["p", "rho", "u", "v", "w"]),
    ("resetF", ["items", "Fx", "Fy", "Fz", "NT"], ["Fx", "Fy", "Fz"]),
    ("set_wall_f", ["items", "neib", "ftmp"], ["ftmp"]),
    ("set_out", ["items", "neib", "ftmp", "fout", "feq", "f", "posx", "posy", "delX", "delY"], ["fout", "feq", "f"]),
    ("set_fin", ["items", "neib", "nextK", "feq", "f"], ["feq", "f"]),
    ("reset_f", ["items", "ftmp", "feq", "f"], ["feq", "f"]),
    ("set_wall_f_inv", ["items", "neib", "nextB", "nextK", "f"], ["f"]),
    ("set_tmp", ["items", "neib", "f", "ftmp", "fout", "feq"], ["ftmp"]),
    ("set_wall_propagation", ["items", 1, "neib", "nextK", "nextB", "ftmp"], ["ftmp"]),
    ("set_wall_propagation", ["items", 0, "neib", "nextK", "nextB", "ftmp"], ["ftmp"]),
    ("propagation", ["items", "neib", "f", "ftmp"], ["f"]),
    ("reset_wall_fin", ["items", "feq", "f"], ["feq", "f"]),
    ("set_wall_rho", ["items", "neib", "rho"], ["rho"]),
    ("reset_pressure", ["items", "p", "f", "u", "v", "w", 2.0], ["p", "f"]),
    ("LES", ["items", "neib", "tau", "taus", "phi", "rho", 1e-5, 1.016e-3, "u", "v", "w", "posx", "posy", "posz"],
     ["tau", "taus"]),
    ("wall_function", ["items", "delX", "delY", 0, 0, 1, "NW5", "w5", "u", "v", "w", "Fx", "Fy", "rho"], ["Fx", "Fy"]),
]


def make_inputs(case_key, prec, seed=7):
    kw = dict(CASES[case_key])
    c = cases.box_case(prec=prec, nu=1e-3, **kw)
    st = random_state(c, seed, tau=0.62, taus=0.57)
    rng = np.random.default_rng(seed + 1)
    dt = c["dtype"]
    Q, nt = c["Q"], c["nt"]
    st = dict(st)
    # distinct random contents for every scratch buffer, ghosts included
    for k in ("ftmp", "fout", "feq", "Fk"):
        st[k] = (1e-3 * rng.standard_normal(nt * Q)).astype(dt)
    for k in ("Fx", "Fy", "Fz"):
        st[k] = (1e-2 * rng.standard_normal(nt)).astype(dt)
    st["phi"] = rng.uniform(0.05, 0.95, nt).astype(dt)
    for k, src in (("phio", "phi"), ("uo", "u"), ("vo", "v"), ("wo", "w")):
        st[k] = (st[src] * (1 + 0.1 * rng.standard_normal(nt))).astype(dt)
    M, Minv, S, MM = mrt_mats(9) if Q == 9 else _q27_mats()
    if M is not None:
        for k, v in (("M", M), ("Minv", Minv), ("S", S), ("MM", MM)):
            st[k] = np.ascontiguousarray(v, dtype=dt).ravel()
    return c, st


def _q27_mats():
    from oracle import oracle as _o
    import os

    if not os.path.exists(os.path.join(_o.REF_INPUT_DIR, "input", "MRT_D3Q27.csv")):
        return None, None, None, None
    from ip_cu_lbm_b200 import _lib

    Q = 27
    M, S, Mi = np.zeros((Q, Q)), np.zeros(Q), np.zeros((Q, Q))
    _lib.check(_lib.lib().ipcu_read_M_csv(_o.REF_INPUT_DIR.encode(), Q, M.ctypes.data, S.ctypes.data, Mi.ctypes.data))
    M2, S2, Mi2, MM = cases.set_M(Q, M, S, Mi)
    return M2, Mi2, S2, MM


def resolve(args, c, bufs):
    out = []
    for a in args:
        if isinstance(a, str):
            if a == "NT":
                out.append(c["nt"])
            elif a == "NW5":
                out.append(len(c["walls"][4]))
            elif a in ("w1", "w2", "w3", "w4", "w5", "w6"):
                out.append(bufs[a])
            else:
                out.append(bufs[a])
        else:
            out.append(a)
    return out


def run_kernel(backend, name, args, c, st, prec):
    import torch

    from ip_cu_lbm_b200 import _lib

    nt = c["nt"]
    tdt = torch.float32 if prec == "f32" else torch.float64
    host = dict(st)
    for k in ("items", "neib", "nextB", "nextK", "posx", "posy", "posz", "delX", "delY"):
        host[k] = c[k]
    for a, wl in enumerate(c["walls"]):
        host[f"w{a + 1}"] = wl if len(wl) else np.zeros(1, np.int32)
    if backend == "oracle":
        from oracle import oracle as _o

        dt = np.float32 if prec == "f32" else np.float64
        bufs = {k: np.ascontiguousarray(v, dtype=dt if np.asarray(v).dtype.kind == "f" else np.int32).copy()
                for k, v in host.items()}
        _o.oracle()(name, prec, *resolve(args, c, bufs))
        return bufs
    dev = torch.device("cuda:0")
    bufs = {k: torch.as_tensor(np.ascontiguousarray(v), device=dev,
                               dtype=tdt if np.asarray(v).dtype.kind == "f" else torch.int32).clone()
            for k, v in host.items()}
    res = resolve(args, c, bufs)
    if backend == "ref":
        from oracle import oracle as _o

        assert _o.ref()(name, prec, *res, n=nt) == 0
    else:
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.legacy()(name, prec, *res, tail=(nt, stream)), name)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in bufs.items()}


def _ref_ok():
    from oracle import oracle as _o

    return _o.ref_available()


@pytest.mark.parametrize("case_key", ["q9", "q9u", "q27"])
@pytest.mark.parametrize("idx", range(len(KERNELS)))
def test_kernel_matches_reference_f32(cuda, case_key, idx):
    name, args, outs = KERNELS[idx]
    if not _ref_ok():
        pytest.skip("reference build (oracle/_ref) not present")
    c, st = make_inputs(case_key, "f32")
    if "M" in args and "M" not in st:
        pytest.skip("Q27 MRT input matrices not present")
    mine = run_kernel("ipcu", name, args, c, st, "f32")
    ref = run_kernel("ref", name, args, c, st, "f32")
    for o in outs:
        err = rel_l2(mine[o], ref[o], floor=1e-30)
        assert err <= 2e-6, (name, o, err)


@pytest.mark.parametrize("case_key", ["q9", "q27"])
@pytest.mark.parametrize("idx", range(len(KERNELS)))
def test_kernel_matches_oracle_f64(cuda, case_key, idx):
    name, args, outs = KERNELS[idx]
    c, st = make_inputs(case_key, "f64")
    if "M" in args and "M" not in st:
        pytest.skip("Q27 MRT input matrices not present")
    mine = run_kernel("ipcu", name, args, c, st, "f64")
    orc = run_kernel("oracle", name, args, c, st, "f64")
    for o in outs:
        err = rel_l2(mine[o], orc[o], floor=1e-300)
        assert err <= 1e-12, (name, o, err)


@pytest.mark.parametrize("slip", [0, 1])
@pytest.mark.parametrize("nsteps", [1, 10, 100])
def test_lockexchange_chain_matches_reference(cuda, slip, nsteps):
    if not _ref_ok():
        pytest.skip("reference build (oracle/_ref) not present")
    c = cases.box_case(prec="f32", **CASES["q9"])
    st = random_state(c, 11, tau=0.6, taus=0.55)
    mats = mrt_mats()
    mine = gpu_chain(c, st, nsteps, "ipcu", slip=slip, mats=mats)
    ref = gpu_chain(c, st, nsteps, "ref", slip=slip, mats=mats)
    nc = c["nc"]
    for k in ("u", "w", "sal", "p"):
        err = rel_l2(mine.__dict__[k][:nc], ref.__dict__[k][:nc], floor=1e-30)
        assert err <= 1e-5, (k, err)


@pytest.mark.parametrize("slip", [0, 1])
def test_lockexchange_chain_matches_oracle_f64(cuda, slip):
    c = cases.box_case(prec="f64", **CASES["q9"])
    st = random_state(c, 12, tau=0.6, taus=0.55)
    mats = mrt_mats()
    mine = gpu_chain(c, st, 20, "ipcu", slip=slip, mats=mats)
    orc = oracle_chain(c, st, 20, slip=slip, mats=mats)
    nc = c["nc"]
    for k in ("u", "w", "sal", "p", "f", "g"):
        a, b = getattr(mine, k), getattr(orc, k)
        n = nc * (c["Q"] if k in ("f", "g") else 1)
        err = rel_l2(a[:n], b[:n], floor=1e-300)
        assert err <= 1e-11, (k, err)
