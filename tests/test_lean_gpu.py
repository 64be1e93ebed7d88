"""The lean flow-only step (FP32, no scalar lattice, uniform S: the S plane
untouched, the velocity planes stored only where a body force acted) against
the full step on identical inputs. The recomputed velocity is bit for bit the
stored one, so the two runs must agree exactly: without a body, with a
settling body (direct steps and graph replay), across batched steps and
uploads, and when a non-uniform S turns the lean step off."""
import numpy as np
import pytest

from ip_cu_lbm_b200 import Sim
from ip_cu_lbm_b200.cases import d2q9_mrt
from ip_cu_lbm_b200.serving import Batch

pytestmark = pytest.mark.gpu

FIELDS = ("f", "ux", "uz", "p", "S")


def flow(nx=96, nz=64, s_uni=0.3, g=1e-4, seed=4):
    """A box with a uniform scalar value, Boussinesq gravity on it and a
    smooth random initial velocity (the populations at its equilibrium)."""
    M, Minv, S = d2q9_mrt()
    kw = dict(q_scalar=0, geometry="uniform", wall="bb", tau=0.6, rho_sal=1e-3, g_bouss=g, M=M, Minv=Minv, S=S)
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) / nx
    z = (np.arange(nz) + 0.5) / nz
    ph = rng.uniform(0, 2 * np.pi, 4)
    ux = 1e-3 * np.sin(2 * np.pi * z[:, None] + ph[0]) * np.cos(2 * np.pi * x[None, :] + ph[1])
    uz = 1e-3 * np.cos(2 * np.pi * x[None, :] + ph[2]) * np.sin(np.pi * z[:, None] + ph[3])
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
    ez = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    eu = ex[:, None, None] * ux[None] + ez[:, None, None] * uz[None]
    f = w[:, None, None] * (3 * eu + 4.5 * eu ** 2 - 1.5 * (ux ** 2 + uz ** 2)[None])
    S0 = np.full((nz, nx), s_uni)

    def make():
        s = Sim(nx, nz, s0=S0.ravel(), **kw)
        s.set_state(f=f, S=S0, ux=ux, uz=uz)
        return s

    return make


def same(a, b):
    for k in FIELDS:
        va, vb = a.get(k), b.get(k)
        assert np.array_equal(va, vb), (k, float(np.abs(va - vb).max()))


def test_lean_is_the_default_where_allowed(cuda):
    s = flow()()
    assert s.lean()
    assert s.bytes_per_cell() == 72
    s.set_lean(False)
    assert not s.lean() and s.bytes_per_cell() == 96
    s.set_lean(True)
    assert s.lean()
    s.close()
    # a scalar lattice or a stretched axis keeps the full step
    M, Minv, S = d2q9_mrt()
    s5 = Sim(32, 16, q_scalar=5, M=M, Minv=Minv, S=S)
    assert not s5.lean()
    with pytest.raises(Exception):
        s5.set_lean(True)
    s5.close()


def test_lean_matches_full_step_without_body(cuda):
    make = flow()
    a, b = make(), make()
    b.set_lean(False)
    assert a.lean() and not b.lean()
    for s in (a, b):
        s.step(7)
        s.step_graph(40, chunk=10)
    same(a, b)
    assert a.status() == 0 and b.status() == 0
    a.close()
    b.close()


@pytest.mark.parametrize("graph", [False, True])
def test_lean_matches_full_step_with_settling_body(cuda, graph):
    M, Minv, S = d2q9_mrt()
    kw = dict(q_scalar=0, geometry="uniform", wall="bb", tau=0.56, rho_sal=0.0, g_bouss=0.0, M=M, Minv=Minv, S=S)
    runs = []
    for lean in (True, False):
        s = Sim(64, 96, **kw)
        s.attach_ellipse(32.0, 60.0, 8.0, 4.0, markers=48, theta=np.pi / 4, rho_s=1.5, gravity=1e-4)
        s.set_lean(lean)
        assert s.lean() == lean
        if graph:
            s.step_graph(120, chunk=20)
        else:
            s.step(120)
        runs.append(s)
    a, b = runs
    assert a.body() == b.body()
    same(a, b)
    assert a.status() == 0 and b.status() == 0
    # the body moved through several tiles' worth of its footprint
    assert abs(a.body()["w"]) > 0
    a.close()
    b.close()


def test_lean_after_batched_steps_and_upload(cuda):
    import torch

    make = flow(seed=7)
    a, b = make(), make()
    b.set_lean(False)
    bt = Batch()
    for s in (a, b):
        s.step(5)
        bt.step([s], 7)  # the batched kernel writes every plane (odd: the other parity's flags)
        s.get("ux")  # a read right after the batch must leave the batch's planes alone
        s.step(9)
    same(a, b)
    # a raw download / upload round trip keeps the lean step on (uniform S)
    N = a.N
    hf = torch.empty(9 * N, dtype=torch.float32, pin_memory=True)
    hm = torch.empty(3 * N, dtype=torch.float32, pin_memory=True)
    for s in (a, b):
        s.download(hf, None, hm)
        s.sync()
        s.upload(hf, None, hm)
        s.step(11)
    assert a.lean()
    same(a, b)
    bt.close()
    a.close()
    b.close()


def test_nonuniform_scalar_turns_lean_off(cuda):
    make = flow(seed=9)
    a, b = make(), make()
    b.set_lean(False)
    S1 = a.get("S")
    S1[:, : S1.shape[1] // 2] += 0.1  # a density step: the gradient force matters now
    for s in (a, b):
        s.step(4)
        s.set_state(S=S1)
    assert not a.lean()
    for s in (a, b):
        s.step(12)
    same(a, b)
    a.close()
    b.close()


def test_push_form_is_the_default_and_matches_the_tile_form(cuda):
    """The push form of the lean step (bounce-back, uniform grid, two-moment
    MRT) against the tile form and the full step, with a settling body that
    crosses tiles (so tiles switch between F0, a recorded body force and
    stored planes), direct steps and graph replay, and a switch of form in
    the middle of the run."""
    M, Minv, S = d2q9_mrt()
    kw = dict(q_scalar=0, geometry="uniform", wall="bb", tau=0.56, rho_sal=1e-3, g_bouss=1e-5, M=M, Minv=Minv, S=S)
    runs = []
    for mode in ("push", "tile", "full", "switch"):
        s = Sim(160, 128, s0=np.full(160 * 128, 0.25), **kw)
        s.attach_ellipse(58.0, 60.0, 8.0, 4.0, markers=48, theta=0.4, rho_s=5.0, gravity=1e-4, u=0.05, w=0.01)
        assert s.lean() and s.push()
        if mode == "tile":
            s.set_push(False)
            assert s.lean() and not s.push()
        if mode == "full":
            s.set_lean(False)
        s.step(37)
        if mode == "switch":
            s.set_push(False)
            s.step_graph(40, chunk=10)
            s.set_push(True)
        else:
            s.step_graph(40, chunk=10)
        s.step_graph(223, chunk=50)
        runs.append(s)
    ref = runs[2]
    assert ref.body()["x"] > 64.0  # the body moved across the tile column boundary at x = 64
    for s in runs[:2] + runs[3:]:
        assert s.body() == ref.body()
        same(s, ref)
        assert s.status() == 0
    for s in runs:
        s.close()
    # slip walls keep the tile form
    s = Sim(64, 32, q_scalar=0, wall="slip", M=M, Minv=Minv, S=S)
    assert s.lean() and not s.push()
    with pytest.raises(Exception):
        s.set_push(True)
    s.close()
