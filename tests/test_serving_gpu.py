"""Continuous-batching serving: requests that arrive while others run join
the batch, admission respects the HBM budget, and every request's result is
the same alone and in the mix (the batched kernel runs each simulation's
tiles with the single-run arithmetic)."""
import numpy as np
import pytest

from ip_cu_lbm_b200 import Sim
from ip_cu_lbm_b200.serving import (Batch, Server, falling_ellipse_request, lock_exchange_request,
                                    rayleigh_taylor_request, request_bytes)

pytestmark = pytest.mark.gpu


def _alone(req, batched):
    s = Sim(req.nx, req.nz, s0=req.s0, **req.kwargs)
    if req.body is not None:
        s.attach_ellipse(**req.body)
    if batched:
        b = Batch()
        b.step([s], req.steps)
        b.close()
    else:
        s.step(req.steps)
    out = {k: s.get(k) for k in ("S", "ux", "uz")}
    if req.body is not None:
        out["body"] = s.body()
    s.close()
    return out


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_results_same_alone_and_in_mix(cuda, storage):
    sizes = [(96, 64, 150), (160, 48, 90), (64, 64, 230), (200, 96, 60), (128, 32, 170)]
    reqs = [lock_exchange_request(i, nx, nz, st, arrival=0.0 if i < 2 else 0.01 * i, storage=storage, seed=i)
            for i, (nx, nz, st) in enumerate(sizes)]
    srv = Server(budget_bytes=1e9, tick_steps=40)
    stats = srv.run(reqs)
    srv.close()
    assert stats["requests"] == len(reqs)
    assert stats["cell_updates"] == sum(r.cells * r.steps for r in reqs)
    for r in srv.done:
        same = _alone(r, batched=True)
        for k in ("S", "ux", "uz"):
            assert np.array_equal(r.result[k], same[k]), (r.rid, k)
        plain = _alone(r, batched=False)
        for k in ("S", "ux", "uz"):
            np.testing.assert_allclose(r.result[k], plain[k], rtol=0, atol=1e-6 * max(1.0, np.abs(plain[k]).max()))


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_mixed_salinity_and_phase_field_batch(cuda, storage):
    """Lock-exchange (salinity) and Rayleigh-Taylor (Allen-Cahn phase field)
    requests served together: each kernel class gets its own launch per step
    and every result equals the request run alone."""
    reqs = [lock_exchange_request(0, 96, 64, 120, storage=storage, seed=0),
            rayleigh_taylor_request(1, 128, 128, 160, storage=storage, seed=1),
            lock_exchange_request(2, 64, 48, 80, arrival=0.01, storage=storage, seed=2),
            rayleigh_taylor_request(3, 64, 96, 100, arrival=0.02, storage=storage, seed=3)]
    srv = Server(budget_bytes=1e9, tick_steps=40)
    stats = srv.run(reqs)
    srv.close()
    assert stats["requests"] == len(reqs)
    for r in srv.done:
        same = _alone(r, batched=True)
        for k in ("S", "ux", "uz"):
            assert np.array_equal(r.result[k], same[k]), (r.rid, k)
        assert np.isfinite(r.result["ux"]).all()


def test_budget_limits_admission(cuda):
    reqs = [lock_exchange_request(i, 128, 64, 50, arrival=0.0) for i in range(4)]
    one = request_bytes(reqs[0])
    srv = Server(budget_bytes=2.5 * one, tick_steps=25)
    srv._admit(0.0)
    assert len(srv.active) == 0  # nothing submitted yet
    for r in reqs:
        srv.submit(r, 0.0)
    srv._admit(0.0)
    assert len(srv.active) == 2 and len(srv.waiting) == 2
    stats = srv.run([])
    srv.close()
    assert stats["requests"] == 4


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_immersed_body_requests_in_the_mix(cuda, storage):
    """Falling-ellipse requests batched with lock-exchange requests: each
    body's one-CTA update runs in one launch per step for all bodies, its
    sums in a fixed order, so every result -- fields and body -- is the
    request's own result run alone, bit for bit."""
    reqs = [falling_ellipse_request(0, 192, 576, 150, storage=storage, seed=0),
            lock_exchange_request(1, 96, 64, 120, storage=storage, seed=1),
            falling_ellipse_request(2, 224, 672, 90, arrival=0.01, storage=storage, seed=2)]
    srv = Server(budget_bytes=2e9, tick_steps=40)
    stats = srv.run(reqs)
    srv.close()
    assert stats["requests"] == len(reqs)
    for r in srv.done:
        same = _alone(r, batched=True)
        for k in ("S", "ux", "uz"):
            assert np.array_equal(r.result[k], same[k]), (r.rid, k)
        if r.body is not None:
            assert r.result["body"] == same["body"]
            assert r.result["body"]["z"] < r.body["zc"]  # the ellipse sinks


def test_request_bytes_match_device_bytes(cuda):
    for r in (lock_exchange_request(0, 96, 64, 10, storage="f16"), rayleigh_taylor_request(1, 64, 96, 10),
              falling_ellipse_request(2, 192, 576, 10), falling_ellipse_request(3, 256, 768, 10, storage="f32")):
        s = Sim(r.nx, r.nz, s0=r.s0, **r.kwargs)
        if r.body is not None:
            s.attach_ellipse(**r.body)
        assert s.device_bytes() == request_bytes(r), (r.rid, s.device_bytes(), request_bytes(r))
        s.close()


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_ragged_step_counts_in_one_call(cuda, storage):
    """ipcu_batch_launch_each: bodies, salinity and phase-field simulations
    with different step counts (one of them 0) in one call. The fluid
    launches that follow a batch of body updates start beside it, and every
    result equals the simulation stepped one synchronised step at a time,
    where nothing overlaps, bit for bit."""
    reqs = [falling_ellipse_request(0, 192, 576, 70, storage=storage, seed=0),
            lock_exchange_request(1, 96, 64, 120, storage=storage, seed=1),
            falling_ellipse_request(2, 224, 672, 33, storage=storage, seed=2),
            rayleigh_taylor_request(3, 128, 128, 0, storage=storage, seed=3),
            lock_exchange_request(4, 64, 48, 57, storage=storage, seed=4),
            rayleigh_taylor_request(5, 64, 96, 91, storage=storage, seed=5)]

    def make(r):
        s = Sim(r.nx, r.nz, s0=r.s0, **r.kwargs)
        if r.body is not None:
            s.attach_ellipse(**r.body)
        return s

    sims = [make(r) for r in reqs]
    b = Batch()
    b.launch_each(sims, [r.steps for r in reqs])
    b.sync()
    with pytest.raises(RuntimeError):
        b.launch_each(sims[:1], [-1])
    b.close()
    for r, s in zip(reqs, sims):
        ref = make(r)
        for _ in range(r.steps):
            ref.step(1)
            ref.sync()  # the next step's launch waits for this one to end
        assert s.steps() == r.steps
        for k in ("S", "ux", "uz"):
            assert np.array_equal(s.get(k), ref.get(k)), (r.rid, k)
        if r.body is not None:
            assert s.body() == ref.body()
        assert s.status() == 0
        ref.close()
        s.close()
