"""x-slab decomposition of one lattice: the reference's BIGLAT scheme
(SU(N)/suncl/suncl.cpp:4004-4062, 4804-5210), which cuts the lattice into
sub-lattices along x and exchanges their boundary links after every update
kernel, here as x-slabs of the C-ABI's slab contexts (qg_set_slab).

A slab of w x-slices is a context of size (w + 2, N2, N3, N4): slices 1..w
are its part of the lattice, slices 0 and w + 1 hold copies of the
neighbours' boundary slices (halos).  qg_phase updates the interior only,
with the whole lattice's parity and Philox thread indices, so the slabs
together draw exactly the numbers the undecomposed lattice draws and, with
the halos refreshed after every phase, follow its chain bit for bit.  After
phase (mu, p) only the links of direction mu and parity p have changed, so
the exchange moves one boundary slice of those links to each side:
3 planes x N2 N3 N4 / 2 links (SU(3)).

  SlabSet   -- several slabs on one GPU (the reference runs BIGLAT's
               sub-lattices on one device the same way to test it,
               QCDGPU.cpp:129-134); halos copied through a device buffer.
  DistSlab  -- one slab per rank (torch.distributed: NCCL between GPUs,
               gloo for the host-side test of the exchange); halos sent with
               batched point-to-point operations.

Both run the sweep of qg_sweep: heatbath phases odd X..T, even X..T, n_or
overrelaxation sweeps in the same order, Gram-Schmidt when due (on every
slab; a halo link is reunitarised to the same bits as its original, so no
exchange follows it).
"""
import numpy as np

import qcdgpu_b200 as Q

PARITY_ORDER = (1, 0)          # odd first, as lattice_simulate


def split(n1, parts):
    """x-slice widths of `parts` slabs of a lattice of n1 slices, as even as
    possible, and their first global slices"""
    if parts < 1 or parts > n1:
        raise ValueError("between 1 and N1 slabs")
    w = [n1 // parts + (1 if k < n1 % parts else 0) for k in range(parts)]
    x0 = [sum(w[:k]) for k in range(parts)]
    return w, x0


def slab_config(cfg, w):
    """the context config of a slab of w slices of the lattice cfg"""
    c = Q.default_config()
    for name, _ in Q.Config._fields_:
        setattr(c, name, getattr(cfg, name))
    c.size[0] = w + 2
    return c


def phase_sequence(n_or):
    """(parity, direction, kind) of one sweep, in qg_sweep's order"""
    seq = [(p, mu, Q.HEATBATH) for p in PARITY_ORDER for mu in range(4)]
    for _ in range(n_or):
        seq += [(p, mu, Q.OVERRELAX) for p in PARITY_ORDER for mu in range(4)]
    return seq


def _rows(cfg):
    """reference-layout planes, row size and x-slice length of cfg's lattice"""
    n = list(cfg.size)
    V = int(np.prod(n))
    a = cfg.row_align if cfg.row_align > 0 else 64
    planes = 12 if cfg.group == 3 else 4
    return planes, (V + a - 1) // a * a, V // n[0]


class _Slab:
    """one slab context and its place in the lattice"""

    def __init__(self, cfg, w, x0):
        self.w, self.x0 = w, x0
        self.cfg = slab_config(cfg, w)
        self.L = Q.Lattice(self.cfg)
        self.L.set_slab(x0, cfg.size[0])
        self.nbytes = self.L.slab_halo_bytes()

    def close(self):
        self.L.close()


def _to_slab(table, gcfg, w, x0, scfg):
    """the slab's reference-layout table (halos included) cut from the
    lattice's (global slices x0-1 .. x0+w, periodic)"""
    planes, rows, ns = _rows(gcfg)
    _, srows, _ = _rows(scfg)
    g = table.reshape(planes, rows, 4)
    n1 = gcfg.size[0]
    s = np.zeros((planes, srows, 4), dtype=table.dtype)
    for k in range(w + 2):
        x = (x0 - 1 + k) % n1
        s[:, k * ns:(k + 1) * ns, :] = g[:, x * ns:(x + 1) * ns, :]
    return s.reshape(-1)


class SlabSet:
    """Several x-slabs of one lattice on the current GPU."""

    def __init__(self, cfg, parts):
        import torch
        self.cfg = cfg
        self.widths, self.x0s = split(cfg.size[0], parts)
        self.slabs = [_Slab(cfg, w, x0) for w, x0 in zip(self.widths, self.x0s)]
        nb = max(s.nbytes for s in self.slabs)
        self.buf_hi = [torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in self.slabs]
        self.buf_lo = [torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in self.slabs]
        self.sweeps_done = 0

    def close(self):
        for s in self.slabs:
            s.close()
        self.slabs = []

    def seed(self, randseries=None):
        for s in self.slabs:
            s.L.seed(randseries)

    def upload(self, table):
        """the lattice's links (reference layout, as Lattice.download gives
        them) into the slabs, halos included"""
        for s in self.slabs:
            s.L.upload(_to_slab(table, self.cfg, s.w, s.x0, s.cfg))
        self._sync()

    def download(self):
        """the lattice's links (reference layout) from the slabs' interiors"""
        planes, rows, ns = _rows(self.cfg)
        out = None
        for s in self.slabs:
            t = s.L.download()
            _, srows, _ = _rows(s.cfg)
            if out is None:
                out = np.zeros((planes, rows, 4), dtype=t.dtype)
            t = t.reshape(planes, srows, 4)
            out[:, s.x0 * ns:(s.x0 + s.w) * ns, :] = t[:, ns:(s.w + 1) * ns, :]
        return out.reshape(-1)

    def _sync(self):
        for s in self.slabs:
            s.L.sync()

    def exchange(self, direction, parity):
        """refresh every halo of the links of (direction, parity)"""
        K = len(self.slabs)
        self._sync()                         # the staging buffers are free again
        for k, s in enumerate(self.slabs):
            s.L.slab_halo2(direction, parity, self.buf_lo[k].data_ptr(), self.buf_hi[k].data_ptr(), True)
        self._sync()
        for k, s in enumerate(self.slabs):
            # low halo <- left neighbour's high boundary, high halo <- right's low
            s.L.slab_halo2(direction, parity, self.buf_hi[(k - 1) % K].data_ptr(),
                           self.buf_lo[(k + 1) % K].data_ptr(), False)

    def fill_halos(self):
        for mu in range(4):
            for p in (0, 1):
                self.exchange(mu, p)

    def phase(self, parity, direction, kind=Q.HEATBATH):
        for s in self.slabs:
            s.L.phase(parity, direction, kind)
        self.exchange(direction, parity)

    def sweep(self, n=1):
        for _ in range(n):
            for p, mu, kind in phase_sequence(self.cfg.n_or):
                self.phase(p, mu, kind)
            self.sweeps_done += 1
            if self.cfg.reunit_every > 0 and self.sweeps_done % self.cfg.reunit_every == 0:
                for s in self.slabs:
                    s.L.reunitarize(self.cfg.reunit_fp64)
        self._sync()

    def action_sums(self):
        """(spatial, temporal) sums of (beta/N)(3N - Re Tr U_p) over the
        lattice: the slabs' x-profiles over their interior slices"""
        tot = np.zeros(2)
        for s in self.slabs:
            tot += s.L.action_profile(0)[1:s.w + 1].sum(axis=0)
        return tot

    def polyakov_sums(self):
        """(Re, Im) sums of the Polyakov loop over the spatial sites"""
        tot = np.zeros(2)
        for s in self.slabs:
            tot += s.L.polyakov_profile(0)[1:s.w + 1].sum(axis=0)
        return tot


class DistSlab:
    """One x-slab per rank of a torch.distributed group (rank k holds slab
    k of split(N1, world)).  `slab` is a _Slab, or any object with the same
    nbytes / L.slab_halo2 / L.slab_phase (L.phase for one rank) /
    L.reunitarize / L.sync (and, for device buffers, L.stream) members (the
    host-side test passes a stand-in)."""

    def __init__(self, cfg, dist, device, slab=None, overlap=None):
        import torch
        self.cfg, self.dist = cfg, dist
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        # split each phase so the swap overlaps the interior (default: when
        # there is a neighbour to swap with)
        self.overlap = self.world > 1 if overlap is None else bool(overlap)
        w, x0 = split(cfg.size[0], self.world)
        self.slab = slab if slab is not None else _Slab(cfg, w[self.rank], x0[self.rank])
        nb = self.slab.nbytes
        self.send_hi, self.send_lo, self.recv_hi, self.recv_lo = (
            torch.empty(nb, dtype=torch.uint8, device=device) for _ in range(4))
        self.comm = torch.cuda.Stream(device=device) if self.send_hi.is_cuda else None
        self.sweeps_done = 0

    def _swap(self):
        """send the packed boundaries, receive the neighbours' (current
        stream)"""
        if self.world == 1:
            self.recv_lo.copy_(self.send_hi)
            self.recv_hi.copy_(self.send_lo)
            return
        right, left = (self.rank + 1) % self.world, (self.rank - 1) % self.world
        P2P = self.dist.P2POp
        ops = [P2P(self.dist.isend, self.send_hi, right), P2P(self.dist.irecv, self.recv_lo, left),
               P2P(self.dist.isend, self.send_lo, left), P2P(self.dist.irecv, self.recv_hi, right)]
        for r in self.dist.batch_isend_irecv(ops):
            r.wait()

    def phase(self, parity, direction, kind):
        """one phase with its halo exchange overlapping the interior update:
        boundary slices, pack, then the interior on the slab's stream while
        the swap runs on a second stream; the halos are unpacked (after the
        swap) before the next phase reads them.  On the host (gloo) the
        steps run in turn."""
        import torch
        L = self.slab.L
        if not self.overlap:                 # one launch, then the exchange
            L.phase(parity, direction, kind)
            self.exchange(direction, parity)
            return
        L.slab_phase(parity, direction, kind, 0)
        L.slab_halo2(direction, parity, self.send_lo.data_ptr(), self.send_hi.data_ptr(), True)
        if self.send_hi.is_cuda:
            ctx = torch.cuda.ExternalStream(L.stream(), device=self.send_hi.device)
            packed = torch.cuda.Event()
            packed.record(ctx)
            L.slab_phase(parity, direction, kind, 1)
            with torch.cuda.stream(self.comm):
                self.comm.wait_event(packed)
                self._swap()
                swapped = torch.cuda.Event()
                swapped.record(self.comm)
            ctx.wait_event(swapped)
        else:
            L.sync()
            L.slab_phase(parity, direction, kind, 1)
            self._swap()
        L.slab_halo2(direction, parity, self.recv_lo.data_ptr(), self.recv_hi.data_ptr(), False)

    def exchange(self, direction, parity):
        """refresh the halos of (direction, parity) without an update"""
        import torch
        L = self.slab.L
        L.slab_halo2(direction, parity, self.send_lo.data_ptr(), self.send_hi.data_ptr(), True)
        if self.send_hi.is_cuda:
            with torch.cuda.stream(torch.cuda.ExternalStream(L.stream(), device=self.send_hi.device)):
                self._swap()
        else:
            L.sync()
            self._swap()
        L.slab_halo2(direction, parity, self.recv_lo.data_ptr(), self.recv_hi.data_ptr(), False)

    def fill_halos(self):
        for mu in range(4):
            for p in (0, 1):
                self.exchange(mu, p)

    def sweep(self, n=1):
        for _ in range(n):
            for p, mu, kind in phase_sequence(self.cfg.n_or):
                self.phase(p, mu, kind)
            self.sweeps_done += 1
            if self.cfg.reunit_every > 0 and self.sweeps_done % self.cfg.reunit_every == 0:
                self.slab.L.reunitarize(self.cfg.reunit_fp64)
        self.slab.L.sync()


def main():
    """torchrun --nproc-per-node N -m qcdgpu_b200.slabs [--size 64] [--sweeps 10]
    one slab per rank of an SU(3) (or SU(2)) lattice from a cold start; rank 0
    prints the sweep time (slowest rank, CUDA events on the slab's stream)
    and the lattice's plaquette and Polyakov loop"""
    import argparse
    import json

    import torch

    from qcdgpu_b200 import replicas as RP
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=32)
    ap.add_argument("--group", type=int, default=3)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--beta", type=float, default=6.0)
    ap.add_argument("--n-or", type=int, default=4)
    ap.add_argument("--sweeps", type=int, default=10)
    ap.add_argument("--seed", type=int, default=54)
    a = ap.parse_args()
    rank, world, local = RP.dist_env()
    torch.cuda.set_device(local)
    import torch.distributed as dist
    if world > 1:
        RP.init("nccl", 300, torch.device("cuda", local))
    else:
        dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0, world_size=1,
                                device_id=torch.device("cuda", local))
    cfg = Q.default_config(group=a.group, size=a.size, precision=a.precision, start=Q.START_COLD,
                           prng=Q.PRNG_PHILOX, beta=a.beta, n_or=a.n_or, reunit_every=10, reunit_fp64=1,
                           randseries=a.seed)
    D = DistSlab(cfg, dist, torch.device("cuda", local))
    L = D.slab.L
    L.seed()
    L.init(Q.START_COLD)
    D.fill_halos()
    D.sweep(1)
    stream = torch.cuda.ExternalStream(L.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    e0.record(stream)
    D.sweep(a.sweeps)
    e1.record(stream)
    e1.synchronize()
    ms = torch.tensor([e0.elapsed_time(e1)], device="cuda")
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    w = D.slab.w
    sums = torch.tensor(np.concatenate([L.action_profile(0)[1:w + 1].sum(axis=0),
                                        L.polyakov_profile(0)[1:w + 1].sum(axis=0)]), device="cuda")
    dist.all_reduce(sums)
    V = a.size ** 4
    N = a.group
    bet = float(np.float32(a.beta / N)) if a.precision == 0 else a.beta / N
    s = sums.cpu().numpy()
    # each plaquette contributes (beta/N)(N - Re Tr): mean Re Tr per plaquette, range [-N, N]
    plaq = (6 * N * V - (s[0] + s[1]) / bet) / (6 * V)
    if rank == 0:
        per = ms.item() / a.sweeps
        print(json.dumps({"workload": "SU(%d) %d^4 beta=%.2f, 1 HB + %d OR, x-slabs over %d ranks"
                                      % (N, a.size, a.beta, a.n_or, world),
                          "ms_per_sweep": per, "link_updates_per_s": 4 * V * (1 + a.n_or) / (per * 1e-3),
                          "plaquette": plaq, "polyakov_re": s[2] / (V / a.size * N), "slab_widths": split(a.size, world)[0]}))
    D.slab.close()
    dist.destroy_process_group()


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


if __name__ == "__main__":
    main()
