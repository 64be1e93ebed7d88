"""Moving immersed boundary on the fused 2-D path (ipcu_sim_ib_attach)
against the FP64 oracle (oracle/ibm2d.py): an ellipse settling from rest,
tilted, in a bounce-back box; FP32 and 16-bit storage; alone, batched and
graph-replayed."""
import numpy as np
import pytest

from ip_cu_lbm_b200 import Sim
from ip_cu_lbm_b200.serving import Batch
from ip_cu_lbm_b200.cases import d2q9_mrt, ellipse_markers
from oracle.ibm2d import Body2D, IBBox
from oracle.structured import Box
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

NX, NZ = 64, 96
A, B = 8.0, 4.0
NM = 48


def case(qs=0, storage="f32", rho_s=1.5, theta=np.pi / 4, grav=1e-4, strat=0.0):
    M, Minv, S = d2q9_mrt()
    kw = dict(q_scalar=qs, geometry="uniform", wall="bb", tau=0.56, taus=0.52, rho_sal=1e-3 if qs else 0.0,
              g_bouss=strat)
    S0 = np.zeros((NZ, NX))
    if qs:
        S0 = 1.0 - (np.arange(NZ)[:, None] + 0.5) / NZ * np.ones((1, NX))  # linear stratification
    sim = Sim(NX, NZ, s0=S0.ravel(), storage=storage, M=M, Minv=Minv, S=S, **kw)
    sim.attach_ellipse(NX / 2, 2 * NZ / 3, A, B, markers=NM, theta=theta, rho_s=rho_s, gravity=grav)
    return sim, (M, Minv, S, kw, S0, rho_s, theta, grav)


def oracle(spec, steps):
    M, Minv, S, kw, S0, rho_s, theta, grav = spec
    b = Box(NX, NZ, M=M, Minv=Minv, S=S, **kw)
    if kw["q_scalar"]:
        b.S = S0.copy()
        b.g = np.array([1 / 3] + [1 / 6] * 4)[:, None, None] * S0[None]
    X0, dS = ellipse_markers(A, B, NM)
    body = Body2D(NX / 2, 2 * NZ / 3, X0, dS, rho_s=rho_s, area=np.pi * A * B, inertia_per_mass=(A * A + B * B) / 4,
                  theta=theta)
    body.a_b = (A, B)
    ib = IBBox(b, body, rho_f=1.0, gravity=grav, iters=3)
    ib.step(steps)
    return b, body


def body_err(d, body):
    ref = np.array([body.X[0], body.X[1], body.U[0], body.U[1], body.th, body.om])
    got = np.array([d["x"], d["z"], d["u"], d["w"], d["theta"], d["omega"]])
    # positions against the distance travelled, velocities against the speed
    dpos = np.abs(got[:2] - ref[:2]).max() / max(np.abs(ref[:2] - [NX / 2, 2 * NZ / 3]).max(), 1e-12)
    dvel = np.abs(got[2:4] - ref[2:4]).max() / np.abs(ref[2:4]).max()
    dth = abs(got[4] - ref[4])
    return dpos, dvel, dth


@pytest.mark.parametrize("qs,rho_s", [(0, 1.5), (0, 1.1), (5, 1.5)])
def test_ib_fp32_matches_oracle(cuda, qs, rho_s):
    steps = 150
    sim, spec = case(qs=qs, rho_s=rho_s, strat=1e-4 if qs else 0.0)
    sim.step(steps)
    assert sim.status() == 0
    b, body = oracle(spec, steps)
    d = sim.body()
    dpos, dvel, dth = body_err(d, body)
    assert dpos < 1e-4 and dvel < 1e-4 and dth < 1e-7, (dpos, dvel, dth)
    eu = rel_l2(sim.get("uz"), b.uz)
    ex = rel_l2(sim.get("ux"), b.ux)
    ef = rel_l2(sim.get("ibfz"), b.fext[1])
    assert eu < 1e-5 and ex < 1e-5 and ef < 1e-4, (eu, ex, ef)
    sim.close()


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_ib_16bit_storage(cuda, storage):
    steps = 150
    sim, spec = case(qs=5, storage=storage, strat=1e-4)
    sim.step(steps)
    assert sim.status() == 0
    b, body = oracle(spec, steps)
    d = sim.body()
    dpos, dvel, dth = body_err(d, body)
    tol = 1e-3 if storage == "f16" else 5e-3
    assert dpos < tol and dvel < tol, (dpos, dvel, dth)
    eu = rel_l2(sim.get("uz"), b.uz)
    assert eu < tol, eu
    sim.close()


def test_ib_rest_state_exact(cuda):
    """A neutrally buoyant body in fluid at rest stays exactly at rest."""
    sim, _ = case(qs=0, rho_s=1.0, grav=1e-3)
    sim.step(40)
    d = sim.body()
    assert d["u"] == 0.0 and d["w"] == 0.0 and d["omega"] == 0.0
    assert d["x"] == NX / 2 and d["z"] == 2 * NZ / 3
    assert np.all(sim.get("ux") == 0.0) and np.all(sim.get("uz") == 0.0)
    sim.close()


def test_ib_graph_and_batch_match_alone(cuda):
    steps = 64
    alone, _ = case(qs=5, strat=1e-4)
    alone.step(steps)
    graph, _ = case(qs=5, strat=1e-4)
    graph.step_graph(steps, chunk=16)
    other, _ = case(qs=5, rho_s=1.1, theta=0.3, strat=1e-4)
    batched, _ = case(qs=5, strat=1e-4)
    plain = Sim(80, 48, q_scalar=5, tau=0.56, taus=0.52)  # a body-free neighbour in the batch
    bt = Batch()
    bt.step([other, batched, plain], steps)
    ref = alone.body()
    for s in (graph, batched):  # the update's sums run in a fixed order: bit for bit
        assert s.body() == ref
        assert np.array_equal(s.get("uz"), alone.get("uz")) and np.array_equal(s.get("ux"), alone.get("ux"))
        assert s.status() == 0
    for s in (alone, graph, other, batched, plain):
        s.close()
    bt.close()


def test_ib_window_overflow_flags_status(cuda):
    """A body whose stencils outgrow the kernel's window is skipped with status bit 8."""
    M, Minv, S = d2q9_mrt()
    sim = Sim(256, 256, q_scalar=0, M=M, Minv=Minv, S=S, tau=0.56)
    sim.attach_ellipse(128, 128, 90.0, 80.0, markers=480, rho_s=1.5, gravity=1e-4)
    sim.step(2)
    assert sim.status() & 8
    d = sim.body()
    assert d["x"] == 128 and d["z"] == 128 and d["w"] == 0.0
    sim.close()


def test_ib_overlap_with_fast_body_matches_serial_order(cuda):
    """A body thrown sideways crosses many tile boundaries. The fluid steps
    that overlap its updates (programmatic dependent launch, each update
    flagging the next footprint in advance) must give exactly what the
    batched path gives, whose launches never overlap."""
    M, Minv, S = d2q9_mrt()
    mk = lambda: Sim(160, 128, q_scalar=0, M=M, Minv=Minv, S=S, tau=0.56)
    sims = [mk() for _ in range(3)]
    for s in sims:
        s.attach_ellipse(58.0, 60.0, A, B, markers=NM, theta=0.4, rho_s=5.0, gravity=1e-4, u=0.05, w=0.01)
    sims[0].step(600)                 # overlapped single steps
    sims[1].step_graph(600, chunk=100)  # overlapped, graph-replayed
    bt = Batch()
    bt.step([sims[2]], 600)           # batched: no overlap
    bt.close()
    ref = sims[2].body()
    assert ref["x"] > 70.0, ref  # its stencils crossed the tile column boundary at x = 64
    for s in sims[:2]:
        assert s.body() == ref
        assert np.array_equal(s.get("ux"), sims[2].get("ux")) and np.array_equal(s.get("uz"), sims[2].get("uz"))
        assert s.status() == 0
    for s in sims:
        s.close()
