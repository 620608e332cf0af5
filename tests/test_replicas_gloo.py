"""The replica path of bench.py on CPU: two gloo ranks (world size 2) run
the coordination code the GPU job runs with NCCL -- distinct chain seeds
per rank, barriers around the timed region, the job time as the slowest
rank's time, the whole-job rate, and the reference arm on rank 0 only."""
import os
import socket

import torch.multiprocessing as mp

from qcdgpu_b200 import replicas as RP


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    dist = RP.init("gloo", timeout_s=60)
    r, w, lr = RP.dist_env()
    RP.barrier(dist)
    t = RP.max_over_ranks(1.0 + 1.5 * rank, dist)          # rank 1 is the slow one
    RP.barrier(dist)
    rate = RP.whole_job_rate(w, 100.0, t)
    out.put((r, w, lr, RP.replica_seed(r), t, rate, RP.reference_arm_runs_here(r)))
    RP.finish(dist)


def test_two_gloo_ranks_coordinate_like_the_gpu_job():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1] and all(x[1] == 2 for x in res)
    assert res[0][3] != res[1][3] and res[0][3] == RP.replica_seed(0)
    assert res[0][4] == res[1][4] == 2.5                    # max over ranks
    assert res[0][5] == res[1][5] == 2 * 100.0 / 2.5
    assert res[0][6] and not res[1][6]


def test_single_process_needs_no_group():
    assert RP.init("gloo") is None
    assert RP.max_over_ranks(3.0, None) == 3.0
    assert RP.whole_job_rate(1, 10.0, 2.0) == 5.0


# ------------------------------------------- beta-scan replica scheduler
from types import SimpleNamespace

from qcdgpu_b200 import betascan as BS


def _fake_runner(ens, idx, a):
    """stands in for a GPU batch: deterministic per-ensemble values, a
    device time proportional to the share's cost"""
    cost = sum(BS.ensemble_cost(ens[k], a.n_or) for k in idx)
    return {"idx": list(idx), "plaquette": [1.0 + 0.01 * k for k in idx], "polyakov_abs": [0.1 * k for k in idx],
            "updates": float(cost * a.sweeps), "ms": cost * 1e-6, "sites": sum(int(sum(ens[k][0])) for k in idx),
            "field_bytes": 0}


def _sched_main(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    dist = RP.init("gloo", timeout_s=60)
    a = SimpleNamespace(n_or=4, sweeps=10)
    ens = BS.workload(13, 54)
    job = BS.schedule(ens, a, dist, rank, world, runner=_fake_runner)
    out.put((rank, job))
    RP.finish(dist)


def test_partition_covers_every_ensemble_once_and_balances():
    ens = BS.workload(64, 54)
    for world in (1, 2, 3, 8, 70):
        sh = BS.partition(ens, world)
        assert sorted(k for s in sh for k in s) == list(range(64))
        assert sh == BS.partition(ens, world)                       # deterministic
        loads = [sum(BS.ensemble_cost(ens[k], 4) for k in s) for s in sh]
        assert max(loads) - min(loads) <= max(BS.ensemble_cost(e, 4) for e in ens)
    assert sum(1 for s in BS.partition(ens, 70) if not s) == 6      # more ranks than ensembles


def test_two_gloo_ranks_run_the_beta_scan_schedule():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sched_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ens = BS.workload(13, 54)
    a = SimpleNamespace(n_or=4, sweeps=10)
    sh = BS.partition(ens, 2)
    for r in (0, 1):
        job = res[r]
        assert job["plaquette"] == [1.0 + 0.01 * k for k in range(13)]      # every ensemble, in order
        assert job["polyakov_abs"] == [0.1 * k for k in range(13)]
        parts = [_fake_runner(ens, s, a) for s in sh]
        assert job["ms"] == max(p["ms"] for p in parts)                       # the slowest rank
        assert job["updates"] == sum(BS.ensemble_cost(e, 4) for e in ens) * 10
        assert abs(job["link_updates_per_s"] - job["updates"] / (job["ms"] * 1e-3)) < 1e-6 * job["link_updates_per_s"]
        assert [x["ensembles"] for x in job["ranks"]] == [len(s) for s in sh]
