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
