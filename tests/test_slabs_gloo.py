"""The multi-GPU x-slab path (qcdgpu_b200.slabs.DistSlab) on CPU: gloo
ranks (world size 2 and 3) run its halo exchange and sweep schedule with a
stand-in slab whose boundary slices carry (rank, direction, parity, side)
marks, so the test sees which boundary reached which halo.  On GPUs the
same code moves the slab context's packed boundary slices over NCCL."""
import ctypes
import os
import socket

import numpy as np
import torch.multiprocessing as mp

NBYTES = 64


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class _FakeL:
    """slab_halo / phase / reunitarize / sync of a slab, on host arrays"""

    def __init__(self, rank):
        self.rank = rank
        self.halo = {}
        self.log = []

    def mark(self, direction, parity, side):
        return np.full(NBYTES, (self.rank * 16 + direction * 4 + parity * 2 + side) % 256, dtype=np.uint8)

    def slab_halo(self, direction, parity, side, ptr, to_buf):
        if to_buf:
            src = self.mark(direction, parity, side)
            ctypes.memmove(ptr, src.ctypes.data, NBYTES)
        else:
            dst = np.zeros(NBYTES, dtype=np.uint8)
            ctypes.memmove(dst.ctypes.data, ptr, NBYTES)
            self.halo[(direction, parity, side)] = int(dst[0]) if np.all(dst == dst[0]) else -1

    def slab_halo2(self, direction, parity, ptr_lo, ptr_hi, to_buf):
        self.slab_halo(direction, parity, 0, ptr_lo, to_buf)
        self.slab_halo(direction, parity, 1, ptr_hi, to_buf)

    def slab_phase(self, parity, direction, kind, part):
        self.log.append(("phase", parity, direction, kind, part))

    def reunitarize(self, fp64):
        self.log.append(("gs", int(bool(fp64))))

    def sync(self):
        pass


class _FakeSlab:
    def __init__(self, rank):
        self.nbytes = NBYTES
        self.L = _FakeL(rank)


def _rank_main(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import torch.distributed as dist

    import qcdgpu_b200 as Q
    from qcdgpu_b200.slabs import DistSlab, phase_sequence
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cfg = Q.default_config(group=3, size=(4 * world, 4, 4, 4), prng=Q.PRNG_PHILOX, n_or=1, reunit_every=2,
                           reunit_fp64=1)
    D = DistSlab(cfg, dist, "cpu", slab=_FakeSlab(rank))
    D.sweep(2)
    seq = [("phase",) + s + (part,) for s in phase_sequence(1) for part in (0, 1)]
    expect = seq + seq + [("gs", 1)]
    out.put((rank, dict(D.slab.L.halo), D.slab.L.log == expect))
    dist.destroy_process_group()


def _run(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def _check(world):
    res = _run(world)
    for rank, halo, log_ok in res:
        assert log_ok, rank
        left, right = (rank - 1) % world, (rank + 1) % world
        for mu in range(4):
            for p in (0, 1):
                # the low halo holds the left neighbour's high boundary, the
                # high halo the right neighbour's low boundary
                assert halo[(mu, p, 0)] == (left * 16 + mu * 4 + p * 2 + 1) % 256, (rank, mu, p)
                assert halo[(mu, p, 1)] == (right * 16 + mu * 4 + p * 2 + 0) % 256, (rank, mu, p)


def test_two_gloo_ranks_exchange_slab_halos():
    _check(2)


def test_three_gloo_ranks_exchange_slab_halos():
    _check(3)
