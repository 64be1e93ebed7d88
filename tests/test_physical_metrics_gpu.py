"""The physical quantities the benchmark configurations are judged by, from
the GPU path in FP32 and in 16-bit storage against the FP64 oracle on the
same inputs:

  * C1 lock exchange (512 x 64, uniform, D2Q9 MRT + D2Q5, g' = 1e-4): the
    gravity-current fronts, where the salinity crosses 1/2 along the bottom
    row (the dense current) and along the top row (the light one);
  * C2 two-layer nonuniform case (1024 x 256, z tanh-stretched): the
    interface height z(S = 1/2) in every column;
  * C3 settling ellipse, scaled down to 160 x 480 with semi-axes 8 x 4 (the
    serving request's shape): settling velocity and angle.

Each run prints its errors (the figures in the design notes come from this
file); the assertions hold them to the accuracy the storage precision allows.
"""
import numpy as np
import pytest

from ip_cu_lbm_b200 import Sim, cases, workloads
from ip_cu_lbm_b200.serving import falling_ellipse_request

pytestmark = pytest.mark.gpu


def crossing(x, s, level=0.5, rightmost=True):
    """Interpolated position where s crosses `level` (the last crossing from
    the left, or the first)."""
    idx = np.nonzero((s[:-1] - level) * (s[1:] - level) <= 0)[0]
    if len(idx) == 0:
        return np.nan
    i = idx[-1] if rightmost else idx[0]
    t = (level - s[i]) / (s[i + 1] - s[i]) if s[i + 1] != s[i] else 0.0
    return x[i] + t * (x[i + 1] - x[i])


def fronts(S):
    x = np.arange(S.shape[1]) + 0.5
    return crossing(x, S[0], rightmost=True), crossing(x, S[-1], rightmost=False)


def _box(params, nx, nz):
    from oracle.structured import Box

    M, Minv, S = cases.d2q9_mrt()
    p = {k: v for k, v in params.items() if k not in ("storage", "s_ref", "mrt")}
    return Box(nx, nz, M=M, Minv=Minv, S=S, **p)


@pytest.fixture(scope="module")
def c1_oracle():
    params, S0, meta = workloads.lock_exchange_uniform()
    b = _box(params, meta["nx"], meta["nz"])
    b.S = S0.copy()
    b.g = np.array([1 / 3] + [1 / 6] * 4)[:, None, None] * S0[None]
    out = {}
    for n in (500, 1000, 1500):
        b.step(500)
        out[n] = fronts(b.S)
    return out


@pytest.mark.parametrize("storage,limit", [("f32", 3e-3), ("f16", 1e-2), ("bf16", 0.1)])
def test_c1_gravity_current_fronts(cuda, c1_oracle, storage, limit):
    params, S0, meta = workloads.lock_exchange_uniform()
    params = dict(params, storage=storage)
    s = Sim(meta["nx"], meta["nz"], s0=S0.ravel(), **params)
    worst = 0.0
    for n in (500, 1000, 1500):
        s.step(500)
        got, ref = fronts(s.get("S")), c1_oracle[n]
        d = max(abs(got[0] - ref[0]), abs(got[1] - ref[1]))
        worst = max(worst, d)
        print(f"C1 {storage} step {n}: fronts {got[0]:.4f}, {got[1]:.4f} cells vs FP64 {ref[0]:.4f}, "
              f"{ref[1]:.4f} (|diff| {d:.2e} cells)")
    # the dense front has travelled from the lock at x = 256
    assert c1_oracle[1500][0] - 256.0 > 10.0
    assert worst <= limit, (storage, worst)
    s.close()


def interface_height(S, z):
    """z(S = 1/2) per column of a stably stratified two-layer field."""
    return np.array([crossing(z, S[:, i], rightmost=False) for i in range(S.shape[1])])


@pytest.fixture(scope="module")
def c2_oracle():
    params, S0, meta = workloads.stratified_nonuniform()
    b = _box(params, meta["nx"], meta["nz"])
    b.S = S0.copy()
    b.g = np.array([1 / 3] + [1 / 6] * 4)[:, None, None] * S0[None]
    b.step(150)
    return interface_height(b.S, params["z"]), b


@pytest.mark.parametrize("storage,limit", [("f32", 1e-4), ("f16", 5e-4), ("bf16", 3e-3)])
def test_c2_interface_height(cuda, c2_oracle, storage, limit):
    ref, b = c2_oracle
    params, S0, meta = workloads.stratified_nonuniform(storage=storage)
    s = Sim(meta["nx"], meta["nz"], s0=S0.ravel(), **params)
    s.step(150)
    got = interface_height(s.get("S"), params["z"])
    d = float(np.nanmax(np.abs(got - ref)))
    moved = float(np.nanmax(np.abs(ref - interface_height(S0, params["z"]))))
    print(f"C2 {storage}: interface height max |diff| {d:.2e} (finest cells) after 150 steps; "
          f"it moved up to {moved:.3e}")
    assert d <= limit, (storage, d)
    s.close()


C3S = dict(nx=160, nz=480, steps=1200)


@pytest.fixture(scope="module")
def c3_oracle():
    from oracle.ibm2d import Body2D, IBBox

    r = falling_ellipse_request(0, C3S["nx"], C3S["nz"], C3S["steps"], storage="f32", seed=3)
    b = _box(dict(r.kwargs, rhoL=1.0, rhoH=1.0, phi=1.0, rho_sal=0.0, g_bouss=0.0, taus=0.52, dz=1.0, dt=1.0),
             r.nx, r.nz)
    bd_ = r.body
    X0, dS = cases.ellipse_markers(bd_["a"], bd_["b"], bd_["markers"])
    bd = Body2D(bd_["xc"], bd_["zc"], X0, dS, rho_s=bd_["rho_s"], area=np.pi * bd_["a"] * bd_["b"],
                inertia_per_mass=(bd_["a"] ** 2 + bd_["b"] ** 2) / 4, theta=bd_["theta"])
    bd.a_b = (bd_["a"], bd_["b"])
    ib = IBBox(b, bd, rho_f=bd_["rho_f"], gravity=bd_["gravity"], iters=bd_["iters"])
    out = {}
    for n in (400, 800, 1200):
        ib.step(400)
        out[n] = (bd.U[1], bd.th)
    return r, out


@pytest.mark.parametrize("storage,limit_w,limit_th", [("f32", 1e-4, 1e-6), ("f16", 1e-4, 1e-6), ("bf16", 1e-3, 1e-5)])
def test_c3_settling_velocity_and_angle(cuda, c3_oracle, storage, limit_w, limit_th):
    r, ref = c3_oracle
    s = Sim(r.nx, r.nz, s0=r.s0, **dict(r.kwargs, storage=storage))
    s.attach_ellipse(**r.body)
    worst_w = worst_th = 0.0
    for n in (400, 800, 1200):
        s.step(400)
        got = s.body()
        dw = abs(got["w"] - ref[n][0]) / abs(ref[n][0])
        dth = abs(got["theta"] - ref[n][1])
        worst_w, worst_th = max(worst_w, dw), max(worst_th, dth)
        print(f"C3 {storage} step {n}: settling velocity {got['w']:.6e} vs FP64 {ref[n][0]:.6e} (rel {dw:.2e}); "
              f"angle {got['theta']:.6f} vs {ref[n][1]:.6f} rad (|diff| {dth:.2e})")
    assert ref[1200][0] < 0  # it sinks
    assert worst_w <= limit_w and worst_th <= limit_th, (storage, worst_w, worst_th)
    s.close()
