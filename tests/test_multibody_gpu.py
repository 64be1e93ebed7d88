"""Several moving immersed boundaries in one simulation (the reference's
IB_index loop over bodies, function/ibm.cu:367-424): two tilted ellipses of
different densities settling side by side in a bounce-back box, against the
multi-body FP64 oracle (oracle/ibm2d.py IBBox with a list of bodies); single
steps, graph replay and the batched path bit for bit; snapshots that resume
bit for bit; the separation rule at attach; the IB CSV of all bodies."""
import numpy as np
import pytest

from ip_cu_lbm_b200 import Sim
from ip_cu_lbm_b200.cases import d2q9_mrt, ellipse_markers
from ip_cu_lbm_b200.serving import Batch
from oracle.ibm2d import Body2D, IBBox
from oracle.structured import Box
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

NX, NZ = 128, 96
A, B, NM = 8.0, 4.0, 48
# (xc, zc, theta, rho_s) of the two bodies
BODIES = [(36.0, 64.0, np.pi / 4, 1.5), (92.0, 58.0, -np.pi / 6, 1.3)]
GRAV = 1e-4


def make(qs=0, storage="f32", strat=0.0, bodies=BODIES):
    M, Minv, S = d2q9_mrt()
    kw = dict(q_scalar=qs, geometry="uniform", wall="bb", tau=0.56, taus=0.52, rho_sal=1e-3 if qs else 0.0,
              g_bouss=strat)
    S0 = np.zeros((NZ, NX))
    if qs:
        S0 = 1.0 - (np.arange(NZ)[:, None] + 0.5) / NZ * np.ones((1, NX))
    sim = Sim(NX, NZ, s0=S0.ravel(), storage=storage, M=M, Minv=Minv, S=S, **kw)
    for xc, zc, th, rs in bodies:
        sim.attach_ellipse(xc, zc, A, B, markers=NM, theta=th, rho_s=rs, gravity=GRAV)
    return sim, (M, Minv, S, kw, S0)


def oracle(spec, steps, bodies=BODIES):
    M, Minv, S, kw, S0 = spec
    b = Box(NX, NZ, M=M, Minv=Minv, S=S, **kw)
    if kw["q_scalar"]:
        b.S = S0.copy()
        b.g = np.array([1 / 3] + [1 / 6] * 4)[:, None, None] * S0[None]
    X0, dS = ellipse_markers(A, B, NM)
    out = []
    for xc, zc, th, rs in bodies:
        bd = Body2D(xc, zc, X0, dS, rho_s=rs, area=np.pi * A * B, inertia_per_mass=(A * A + B * B) / 4, theta=th)
        bd.a_b = (A, B)
        out.append(bd)
    IBBox(b, out, rho_f=1.0, gravity=GRAV, iters=3).step(steps)
    return b, out


@pytest.mark.parametrize("qs", [0, 5])
def test_two_bodies_match_oracle(cuda, qs):
    steps = 150
    sim, spec = make(qs=qs, strat=1e-4 if qs else 0.0)
    assert sim.n_bodies == 2
    sim.step(steps)
    assert sim.status() == 0
    b, ref = oracle(spec, steps)
    for i, (bd, (xc, zc, _, _)) in enumerate(zip(ref, BODIES)):
        d = sim.body(i)
        got = np.array([d["x"], d["z"], d["u"], d["w"], d["theta"], d["omega"]])
        want = np.array([bd.X[0], bd.X[1], bd.U[0], bd.U[1], bd.th, bd.om])
        dpos = np.abs(got[:2] - want[:2]).max() / np.abs(want[:2] - [xc, zc]).max()
        dvel = np.abs(got[2:4] - want[2:4]).max() / np.abs(want[2:4]).max()
        dth = abs(got[4] - want[4])
        print(f"body {i}: w {d['w']:.6e} vs FP64 {bd.U[1]:.6e}; position rel {dpos:.2e}, velocity rel {dvel:.2e}, "
              f"angle {dth:.2e}")
        assert want[3] < 0  # it sinks
        assert dpos < 1e-4 and dvel < 1e-4 and dth < 1e-7, (i, dpos, dvel, dth)
    eu, ex = rel_l2(sim.get("uz"), b.uz), rel_l2(sim.get("ux"), b.ux)
    ef = rel_l2(sim.get("ibfz"), b.fext[1])
    assert eu < 1e-5 and ex < 1e-5 and ef < 1e-4, (eu, ex, ef)
    # the bodies differ: different densities settle at different speeds
    assert abs(sim.body(0)["w"] - sim.body(1)["w"]) > 0.1 * abs(sim.body(1)["w"])
    sim.close()


def test_two_bodies_graph_and_batch_match_single_steps(cuda):
    steps = 64
    alone, _ = make(qs=5, strat=1e-4)
    alone.step(steps)
    graph, _ = make(qs=5, strat=1e-4)
    graph.step_graph(steps, chunk=16)
    batched, _ = make(qs=5, strat=1e-4)
    one, _ = make(qs=5, strat=1e-4, bodies=BODIES[:1])  # a one-body neighbour in the batch
    plain = Sim(80, 48, q_scalar=5, tau=0.56, taus=0.52)
    bt = Batch()
    bt.step([one, batched, plain], steps)
    bt.close()
    for s in (graph, batched):
        for i in range(2):
            assert s.body(i) == alone.body(i)
        for fld in ("ux", "uz", "ibfx", "ibfz"):
            assert np.array_equal(s.get(fld), alone.get(fld)), fld
        assert s.status() == 0
    for s in (alone, graph, batched, one, plain):
        s.close()


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_two_bodies_restore_bit_identically(cuda, tmp_path, storage):
    """The snapshot holds every body (description, rigid-body state with its
    previous orientation, footprints, tile flags, marker forces) and the
    shared force density."""
    a, _ = make(storage=storage)
    a.step(40)
    snap = tmp_path / "two.ipcu"
    a.save(snap)
    a.step(30)
    b = Sim.load(snap)
    assert b.steps() == 40 and b.n_bodies == 2
    b.step(30)
    for i in range(2):
        assert a.body(i) == b.body(i)
        assert np.array_equal(a.markers(i), b.markers(i))
    for fld in ("f", "ux", "uz", "ibfx", "ibfz"):
        assert np.array_equal(a.get(fld), b.get(fld)), fld
    assert a.status() == 0 and b.status() == 0


def test_attach_refuses_overlapping_body(cuda):
    sim, _ = make(bodies=BODIES[:1])
    with pytest.raises(RuntimeError):  # outline 4 cells from the first body's
        sim.attach_ellipse(BODIES[0][0] + 2 * A + 4.0, BODIES[0][1], A, B, markers=NM)
    assert sim.n_bodies == 1
    sim.attach_ellipse(BODIES[0][0] + 2 * A + 8.0, BODIES[0][1], A, B, markers=NM)
    assert sim.n_bodies == 2
    with pytest.raises(RuntimeError):
        sim.body(2)
    sim.close()


def test_ib_csv_holds_every_body(cuda, tmp_path):
    sim, _ = make()
    sim.step(20)
    path = tmp_path / "ib.csv"
    sim.write_ib_csv(path)
    rows = np.loadtxt(path, delimiter=",", skiprows=1)
    assert rows.shape == (2 * NM, 9)
    for i in range(2):
        m = sim.markers(i)
        np.testing.assert_allclose(rows[i * NM:(i + 1) * NM], m, rtol=1e-5, atol=1e-12)
        d = sim.body(i)
        assert abs(m[:, 8].sum() - d["Fz"]) <= 1e-5 * np.abs(m[:, 8]).sum() + 1e-15
    sim.close()
