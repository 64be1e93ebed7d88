"""The fused structured-grid solver (ipcu_sim_*) against
  * the reference's own CUDA build running the LockExchange kernel chain on
    the same box (reference layouts: Q9 scalar, x refinement, bounce-back and
    slip), rel-L2 <= 1e-5 in FP32;
  * the FP64 structured oracle on every variant (D2Q5, 3-point upwind, z
    stretching), rel-L2 <= 1e-5 in FP32 storage and <= 1e-3 in FP16 storage;
plus the exact rest state and conservation on the device."""
import numpy as np
import pytest

from ip_cu_lbm_b200 import Sim, cases
from ip_cu_lbm_b200.sim import REF_G_BOUSS, REF_RHO_SAL
from helpers import gpu_chain, mrt_mats, oracle_chain, random_state, rel_l2
from oracle.structured import Box

pytestmark = pytest.mark.gpu

REF_PHYS = dict(rhoL=1.0, rhoH=1000.0, phi=1.0, rho_sal=REF_RHO_SAL, g_bouss=REF_G_BOUSS)


def sim_from_case(c, st, *, slip, storage="f32"):
    NX, nz, nc, Q = c["NX"], c["nz"], c["nc"], c["Q"]
    xs = c["posx"][:nc].reshape(NX, nz)[:, 0].astype(float)
    wx = c["delX"][:nc].reshape(NX, nz)[:, 0].astype(float)
    geo = "uniform" if np.allclose(wx, c["items"][0]) else "x5"
    M, Minv, S = cases.d2q9_mrt()
    s = Sim(NX, nz, q_scalar=9, geometry=geo, storage=storage, wall="slip" if slip == 0 else "bb", mrt=True,
            dz=float(c["items"][0]), dt=float(c["items"][1]), x=xs, wx=wx, tau=float(st["tau"][0]),
            taus=float(st["taus"][0]), M=M, Minv=Minv, S=S, s_ref=0.5, **REF_PHYS)
    grid = lambda a: cases.compact_to_grid(c, a)
    f = st["f"].reshape(-1, Q)[:nc]
    g = st["g"].reshape(-1, Q)[:nc]
    s.set_state(f=np.stack([grid(f[:, k]) for k in range(9)]), g=np.stack([grid(g[:, k]) for k in range(9)]),
                S=grid(st["sal"]), ux=grid(st["u"]), uz=grid(st["w"]))
    return s


LAYOUTS = [dict(nx0=24, nz=10, divx=None),
           dict(nx0=14, nz=9, divx=[1, 1, 2, 4, 2, 1, 1, 1, 2, 2, 1, 1, 1, 1], ratiox=4.0),
           dict(nx0=70, nz=20, divx=None)]


def _ref_ok():
    from oracle import oracle as _o

    return _o.ref_available()


@pytest.mark.parametrize("lay", LAYOUTS)
@pytest.mark.parametrize("slip", [0, 1])
@pytest.mark.parametrize("nsteps", [1, 10, 100])
def test_fused_matches_reference_build(cuda, lay, slip, nsteps):
    if not _ref_ok():
        pytest.skip("reference build (oracle/_ref) not present")
    c = cases.box_case(prec="f32", **lay)
    st = random_state(c, 21, tau=0.6, taus=0.55)
    ref = gpu_chain(c, st, nsteps, "ref", slip=slip, mats=mrt_mats())
    s = sim_from_case(c, st, slip=slip)
    s.step(nsteps)
    grid = lambda a: cases.compact_to_grid(c, a)
    for name, field in (("u", "ux"), ("w", "uz"), ("sal", "S"), ("p", "p")):
        err = rel_l2(s.get(field), grid(getattr(ref, name)), floor=1e-30)
        assert err <= 1e-5, (name, err)
    assert s.status() == 0


@pytest.mark.parametrize("slip", [0, 1])
def test_fused_matches_oracle_chain_f64(cuda, slip):
    c = cases.box_case(prec="f64", **LAYOUTS[1])
    st = random_state(c, 22, tau=0.6, taus=0.55)
    orc = oracle_chain(c, st, 30, slip=slip, mats=mrt_mats())
    s = sim_from_case(c, st, slip=slip)
    s.step(30)
    grid = lambda a: cases.compact_to_grid(c, a)
    for name, field in (("u", "ux"), ("w", "uz"), ("sal", "S")):
        err = rel_l2(s.get(field), grid(getattr(orc, name)), floor=1e-30)
        assert err <= 1e-5, (name, err)


def variant(geo, nx=40, nz=24, seed=5):
    kw = {}
    rng = np.random.default_rng(seed)
    if geo[0] == "x":
        wx = 1.0 + 1.5 * rng.uniform(0, 1, nx)
        kw = dict(x=np.cumsum(wx) - wx / 2, wx=wx)
    if geo[0] == "z":
        xi = (np.arange(nz) + 0.5) / nz
        zh = xi - (0.812 / 2.0) * np.tanh(2.0 * (xi - 0.6))
        zn = zh / zh[-1] * nz * 2.0
        wz = np.gradient(zn)
        wz = wz / wz.min()
        kw = dict(z=np.cumsum(wz) - wz / 2, wz=wz)
    return kw


def init_state(b, seed):
    rng = np.random.default_rng(seed)
    nz, nx = b.nz, b.nx
    xx, zz = np.meshgrid(np.arange(nx), np.arange(nz))
    S = 0.5 + 0.4 * np.sin(2 * np.pi * xx / nx) * np.cos(np.pi * zz / nz)
    u = 1e-3 * np.sin(2 * np.pi * zz / nz)
    w = 1e-3 * np.cos(2 * np.pi * xx / nx)
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])[:, None, None]
    ez = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])[:, None, None]
    w9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)[:, None, None]
    eu = ex * u + ez * w
    f = w9 * (3 * eu + 4.5 * eu ** 2 - 1.5 * (u * u + w * w)) + 1e-5 * w9 * rng.standard_normal((9, nz, nx))
    q = b.qs
    wq = (np.array([1 / 3] + [1 / 6] * 4) if q == 5 else w9[:, 0, 0])[:, None, None]
    g = wq * S * (1 + 3 * eu[:q])
    return f, g, S, u, w


@pytest.mark.parametrize("geo", ["uniform", "x5", "x3", "z5", "z3"])
@pytest.mark.parametrize("qs", [5, 9])
@pytest.mark.parametrize("wall", ["bb", "slip"])
def test_fused_matches_structured_oracle(cuda, geo, qs, wall):
    M, Minv, S = cases.d2q9_mrt()
    nx, nz = 40, 24
    kw = variant(geo, nx, nz)
    phys = dict(tau=0.56, taus=0.52, rhoL=1.0, rhoH=1.0, phi=1.0, rho_sal=1e-3, g_bouss=1e-4)
    b = Box(nx, nz, q_scalar=qs, geometry=geo, wall=wall, M=M, Minv=Minv, S=S, **phys, **kw)
    f, g, Sc, u, w = init_state(b, 1)
    b.f, b.g, b.S, b.ux, b.uz = f.copy(), g.copy(), Sc.copy(), u.copy(), w.copy()
    s = Sim(nx, nz, q_scalar=qs, geometry=geo, wall=wall, M=M, Minv=Minv, S=S, **phys, **kw)
    s.set_state(f=f, g=g, S=Sc, ux=u, uz=w)
    for n in (1, 20):
        b.step(n)
        s.step(n)
    for name, mine, ref in (("ux", s.get("ux"), b.ux), ("uz", s.get("uz"), b.uz), ("S", s.get("S"), b.S)):
        err = rel_l2(mine, ref)
        assert err <= 1e-5, (name, err)


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_reduced_precision_storage_error(cuda, storage):
    """FP16 and BF16 storage with FP32 arithmetic stay within 1e-3 rel-L2 of
    the FP64 oracle on the nonuniform (z-stretched, 3-point upwind) case."""
    M, Minv, S = cases.d2q9_mrt()
    nx, nz = 64, 32
    kw = variant("z3", nx, nz)
    phys = dict(tau=0.56, taus=0.52, rhoL=1.0, rhoH=1.0, phi=1.0, rho_sal=1e-3, g_bouss=1e-4)
    b = Box(nx, nz, q_scalar=5, geometry="z3", wall="bb", M=M, Minv=Minv, S=S, **phys, **kw)
    f, g, Sc, u, w = init_state(b, 2)
    b.f, b.g, b.S, b.ux, b.uz = f.copy(), g.copy(), Sc.copy(), u.copy(), w.copy()
    s = Sim(nx, nz, q_scalar=5, geometry="z3", storage=storage, s_ref=0.5, M=M, Minv=Minv, S=S, **phys, **kw)
    s.set_state(f=f, g=g, S=Sc, ux=u, uz=w)
    b.step(200)
    s.step(200)
    eu = rel_l2(np.stack([s.get("ux"), s.get("uz")]), np.stack([b.ux, b.uz]))
    es = rel_l2(s.get("S"), b.S)
    print(f"{storage} storage, 200 steps: velocity {eu:.2e}, salinity {es:.2e}")
    assert eu <= 1e-3 and es <= 1e-3, (eu, es)


def test_rest_state_exact(cuda):
    nx, nz = 50, 30
    kw = variant("z5", nx, nz)
    s = Sim(nx, nz, q_scalar=5, geometry="z5", g_bouss=0.0, rho_sal=0.0, s0=np.full(nx * nz, 0.3), **kw)
    s.step(50)
    assert not np.any(s.get("f")) and not np.any(s.get("ux")) and not np.any(s.get("uz"))
    assert np.all(np.abs(s.get("S") - 0.3) <= 2e-7)


def test_mass_and_salinity_conserved_on_device(cuda):
    nx, nz = 128, 64
    S0 = np.where(np.arange(nx)[None, :] < nx // 2, 1.0, 0.0) * np.ones((nz, 1))
    s = Sim(nx, nz, q_scalar=5, geometry="uniform", g_bouss=1e-4, rho_sal=1e-4, tau=0.53, taus=0.503,
            s0=S0.ravel())
    p0, s0 = s.totals()
    s.step(500)
    p1, s1 = s.totals()
    # FP32 storage: round-off of ~1 ulp per cell and step accumulates
    assert abs(s1 - s0) <= 1e-4 * s0
    assert abs(p1 - p0) <= 1e-6 * nx * nz
    assert s.status() == 0


def test_graph_replay_equals_direct_steps(cuda):
    nx, nz = 100, 40
    S0 = (np.arange(nx)[None, :] < 50) * np.ones((nz, 1))
    a = Sim(nx, nz, s0=S0.ravel())
    b = Sim(nx, nz, s0=S0.ravel())
    a.step(70)
    b.step_graph(70, chunk=16)
    for fld in ("f", "g", "S", "ux", "uz"):
        assert np.array_equal(a.get(fld), b.get(fld)), fld
