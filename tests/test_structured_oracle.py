"""The numpy structured-grid oracle (oracle/structured.py) agrees with the
kernel-by-kernel oracle chain (oracle/ipcu_oracle.cpp, itself pinned to the
reference build) on the reference's own layouts: rectangular x-z boxes with
x refinement, Q9 scalar, bounce-back and slip walls, MRT. FP64, <= 1e-12."""
import numpy as np
import pytest

from ip_cu_lbm_b200 import cases
from helpers import mrt_mats, oracle_chain, random_pf_state, random_state, rel_l2
from oracle.structured import Box

BOXES = [
    dict(nx0=9, nz=6, divx=None),
    dict(nx0=7, nz=5, divx=[1, 2, 3, 1, 2, 1, 1]),
    dict(nx0=3, nz=4, divx=[2, 3, 1]),
]


def structured_from_case(c, st, *, slip, mats, qs=9, **phys):
    NX, nz, nc, Q = c["NX"], c["nz"], c["nc"], c["Q"]
    xs = c["posx"][:nc].reshape(NX, nz)[:, 0].astype(float)
    wx = c["delX"][:nc].reshape(NX, nz)[:, 0].astype(float)
    geo = "uniform" if np.allclose(wx, c["items"][0]) else "x5"
    M, Minv, S, _ = mats
    b = Box(NX, nz, q_scalar=qs, geometry=geo, wall="slip" if slip == 0 else "bb", mrt=True, dz=float(c["items"][0]),
            dt=float(c["items"][1]), x=xs, wx=wx, tau=float(st["tau"][0]), taus=float(st["taus"][0]),
            M=M, Minv=Minv, S=np.ones(9), **phys)
    grid = lambda a: cases.compact_to_grid(c, a)
    f = st["f"].reshape(-1, Q)[:nc]
    g = st["g"].reshape(-1, Q)[:nc]
    b.f = np.stack([grid(f[:, k]) for k in range(9)]).astype(float)
    b.g = np.stack([grid(g[:, k]) for k in range(qs)]).astype(float)
    b.S, b.ux, b.uz = grid(st["sal"]), grid(st["u"]), grid(st["w"])
    return b


@pytest.mark.parametrize("bx", BOXES)
@pytest.mark.parametrize("slip", [0, 1])
@pytest.mark.parametrize("nsteps", [1, 6])
def test_structured_oracle_matches_kernel_chain(bx, slip, nsteps):
    c = cases.box_case(prec="f64", nx0=bx["nx0"], nz=bx["nz"], divx=bx["divx"])
    st = random_state(c, 3 + nsteps, tau=0.63, taus=0.58)
    mats = mrt_mats()
    chain = oracle_chain(c, st, nsteps, slip=slip, mats=mats)
    b = structured_from_case(c, st, slip=slip, mats=mats, rhoL=1.0, rhoH=1000.0, phi=1.0, rho_sal=0.824493,
                             g_bouss=0.824493 * 9.81)
    b.step(nsteps)
    grid = lambda a: cases.compact_to_grid(c, a)
    for name, mine, ref in (("u", b.ux, chain.u), ("w", b.uz, chain.w), ("S", b.S, chain.sal), ("p", b.p, chain.p)):
        err = rel_l2(mine, grid(ref), floor=1e-300)
        assert err <= 1e-12, (name, err)
    f = chain.f.reshape(-1, 9)[: c["nc"]]
    err = rel_l2(b.f, np.stack([grid(f[:, k]) for k in range(9)]))
    assert err <= 1e-12, ("f", err)


PF_PHYS = dict(rhoL=1.0, rhoH=3.0)


@pytest.mark.parametrize("bx", BOXES)
@pytest.mark.parametrize("slip", [0, 1])
@pytest.mark.parametrize("nsteps", [1, 6])
def test_structured_phase_field_matches_kernel_chain(bx, slip, nsteps):
    """Two-phase (Allen-Cahn) mode against the reference's two-phase kernel
    order on the oracle chain: surface tension, the mixture's weight,
    col_PF with its d(phi u)/dt term. The reference fixes tau_phi = 0.58."""
    c = cases.box_case(prec="f64", nx0=bx["nx0"], nz=bx["nz"], divx=bx["divx"], dx=1e-3, dt=1e-4, sigma=2e-4)
    st = random_pf_state(c, 11 + nsteps, tau=0.63, taus=0.58, **PF_PHYS)
    mats = mrt_mats()
    chain = oracle_chain(c, st, nsteps, slip=slip, mats=mats, kind="pf", **PF_PHYS)
    st_b = dict(st)
    st_b["sal"] = st["phi"]
    it = c["items"]
    b = structured_from_case(c, st_b, slip=slip, mats=mats, phase_field=True, sigma=float(it[16]),
                             pf_width=float(it[9]), gravity=9.81, **PF_PHYS)
    b.old = np.stack([b.S * b.ux, b.S * b.uz])
    b.step(nsteps)
    grid = lambda a: cases.compact_to_grid(c, a)
    for name, mine, ref in (("u", b.ux, chain.u), ("w", b.uz, chain.w), ("phi", b.S, chain.phi), ("p", b.p, chain.p)):
        err = rel_l2(mine, grid(ref), floor=1e-300)
        assert err <= 1e-12, (name, err)


def test_uniform_streaming_is_an_exact_shift():
    """On a uniform axis the flux-form weights are (0,0,1,0,0): the pass is a shift (ref: adv.cu:76-87)."""
    b = Box(6, 5, q_scalar=5, geometry="x5", mrt=False, tau=1.0, taus=1.0)
    assert np.array_equal(b.W[:, :, 2], np.ones((2, 6)))
    assert not np.any(b.W[:, :, [0, 1, 3, 4]])


def test_rest_state_is_preserved_exactly():
    M, Minv, S = cases.d2q9_mrt()
    b = Box(8, 6, q_scalar=5, geometry="z3", z=np.cumsum(np.linspace(1, 2, 6)) - 0.5, wz=np.linspace(1, 2, 6),
            M=M, Minv=Minv, S=S, g_bouss=0.0)
    b.S[:] = 0.25
    b.g[:] = (np.array([1 / 3] + [1 / 6] * 4) * 0.25)[:, None, None]
    b.step(5)
    assert not np.any(b.f) and not np.any(b.ux) and not np.any(b.uz)
    np.testing.assert_allclose(b.S, 0.25, rtol=0, atol=1e-15)


@pytest.mark.parametrize("geo", ["uniform", "x5", "x3", "z5", "z3"])
@pytest.mark.parametrize("wall", ["bb", "slip"])
def test_conservation(geo, wall):
    """Salinity (D2Q5, no diagonals) is conserved to round-off on every grid
    and wall; p* is conserved to round-off on uniform grids and with slip
    walls. With bounce-back on a stretched axis the reference scheme returns
    a diagonal population through the interpolated flux of its partner, which
    is not mass-neutral; the kernel-chain oracle shows the same drift."""
    M, Minv, S = cases.d2q9_mrt()
    nx, nz = 12, 9
    kw = {}
    if geo[0] == "x":
        wx = np.linspace(1, 2.2, nx)
        kw = dict(x=np.cumsum(wx) - wx / 2, wx=wx)
    if geo[0] == "z":
        wz = np.linspace(1, 2.2, nz)
        kw = dict(z=np.cumsum(wz) - wz / 2, wz=wz)
    b = Box(nx, nz, q_scalar=5, geometry=geo, wall=wall, M=M, Minv=Minv, S=S, g_bouss=1e-3, **kw)
    rng = np.random.default_rng(0)
    b.f = 1e-3 * rng.standard_normal((9, nz, nx)) * np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)[:, None, None]
    b.S = rng.uniform(0, 1, (nz, nx))
    b.g = np.array([1 / 3] + [1 / 6] * 4)[:, None, None] * b.S[None]
    area = np.outer(b.DZ, b.DX)
    p0, s0 = (b.f.sum(0) * area).sum(), (b.S * area).sum()
    b.step(20)
    assert abs((b.S * area).sum() - s0) <= 1e-13 * area.sum()
    dp = abs((b.p * area).sum() - p0)
    if geo == "uniform" or wall == "slip":
        assert dp <= 1e-15 * area.sum()
    else:
        assert dp <= 1e-3 * area.sum()
