"""The multi-GPU replica path (one process per GPU, barrier + max-over-ranks
timing, no data collective) exercised with world_size 2 on the gloo backend
on CPU: every rank takes the same collective steps, the aggregate counts all
ranks' work over the slowest rank's time, and a rank that fails to join ends
the others' barrier with an error within the process-group timeout."""
import os
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = textwrap.dedent("""
    import json, os, sys, time
    sys.path.insert(0, %r)
    from ip_cu_lbm_b200.replicas import Replicas
    R = Replicas(backend="gloo", timeout_s=20)
    R.barrier()
    t0 = time.perf_counter()
    time.sleep(0.05 * (R.rank + 1))          # the ranks' independent work
    R.barrier()
    dt = R.max(time.perf_counter() - t0)
    agg = R.aggregate(1000.0, dt)
    if R.rank == 0:
        print(json.dumps({"world": R.world, "dt": dt, "agg": agg}))
    R.close()
""") % ROOT


def _run(n, env_extra=None):
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(29500 + os.getpid() % 1000))
    env.update(env_extra or {})
    procs = []
    for r in range(n):
        e = dict(env, RANK=str(r), WORLD_SIZE=str(n), LOCAL_RANK=str(r))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=e, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=120) for p in procs]
    return procs, outs


def test_two_replicas_max_over_ranks():
    import json

    procs, outs = _run(2)
    assert all(p.returncode == 0 for p in procs), [o[1][-500:] for o in outs]
    line = json.loads(outs[0][0].strip().splitlines()[-1])
    assert line["world"] == 2
    assert line["dt"] >= 0.1  # the slower rank's time
    assert abs(line["agg"] - 2 * 1000.0 / line["dt"]) < 1e-6


def test_missing_rank_ends_with_an_error():
    # only rank 0 of a world of 2 starts: its rendezvous/barrier must fail, not hang
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(30500 + os.getpid() % 1000), RANK="0",
               WORLD_SIZE="2", LOCAL_RANK="0")
    code = WORKER.replace("timeout_s=20", "timeout_s=5")
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=180)
    assert p.returncode != 0
