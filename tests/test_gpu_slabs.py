"""x-slab decomposition (qg_set_slab, qcdgpu_b200.slabs.SlabSet): a lattice
cut into x-slabs on one GPU -- the way the reference exercises its BIGLAT
decomposition on a single device -- follows the undecomposed lattice's
chain bit for bit through heatbath, overrelaxation and Gram-Schmidt, and
the slabs' interior x-profiles add up to the lattice's action and Polyakov
sums."""
import numpy as np
import pytest

import qcdgpu_b200 as Q
from qcdgpu_b200.slabs import DistSlab, SlabSet, _Slab, _to_slab, split

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("group,precision,dims,parts", [
    (3, 0, (8, 4, 4, 6), 2), (3, 0, (8, 4, 4, 6), 3), (3, 1, (6, 4, 2, 4), 2), (3, 0, (4, 4, 4, 4), 3),
    (2, 1, (8, 4, 4, 4), 4), (2, 0, (6, 2, 4, 4), 1)])
def test_slabs_follow_the_whole_lattice_bit_for_bit(group, precision, dims, parts):
    cfg = Q.default_config(group=group, size=dims, precision=precision, start=Q.START_HOT, prng=Q.PRNG_PHILOX,
                           beta=5.8 if group == 3 else 2.3, n_or=2, reunit_every=2, reunit_fp64=1, randseries=77)
    G = Q.Lattice(cfg)
    G.seed()
    G.init(Q.START_HOT)
    S = SlabSet(cfg, parts)
    S.seed()
    S.upload(G.download())
    assert np.array_equal(S.download(), G.download())
    for s in range(3):
        G.sweep(1)
        S.sweep(1)
        assert np.array_equal(S.download(), G.download()), s
    ga, sa = np.array(G.action_sums()), S.action_sums()
    assert np.all(np.abs(sa - ga) <= 1e-12 * np.abs(ga)), (sa, ga)
    gp, sp = np.array(G.polyakov_sums()[:2]), S.polyakov_sums()
    assert np.all(np.abs(sp - gp) <= 1e-12 * (1 + np.abs(gp))), (sp, gp)
    S.close()
    G.close()


def test_slab_halo_fill_from_a_cold_start_and_argument_checks():
    cfg = Q.default_config(group=3, size=(6, 4, 4, 4), precision=0, start=Q.START_COLD, prng=Q.PRNG_PHILOX,
                           beta=6.0, n_or=1, reunit_every=0, randseries=5)
    G = Q.Lattice(cfg)
    G.seed()
    G.init(Q.START_COLD)
    S = SlabSet(cfg, 2)
    S.seed()
    for s in S.slabs:
        s.L.init(Q.START_COLD)
    S.fill_halos()
    S.sweep(2)
    G.sweep(2)
    assert np.array_equal(S.download(), G.download())
    L = S.slabs[0].L
    with pytest.raises(Q.QGError):
        L.sweep(1)                                   # a slab sweeps through the slab driver
    with pytest.raises(Q.QGError):
        L.init(Q.START_HOT)                          # hot / Haar starts are whole-lattice
    host = np.zeros(S.slabs[0].nbytes, dtype=np.uint8)
    with pytest.raises(Q.QGError):                   # the one-launch form takes device buffers only
        L.slab_halo2(0, 0, host.ctypes.data, host.ctypes.data, True)
    S.close()
    G.close()
    with pytest.raises(Q.QGError):                   # RANLUX: no slabs
        Q.Lattice(Q.default_config(group=3, size=(4, 4, 4, 4), prng=Q.PRNG_RANLUX)).set_slab(0, 8)
    with pytest.raises(Q.QGError):                   # odd global N1
        Q.Lattice(Q.default_config(group=3, size=(4, 4, 4, 4), prng=Q.PRNG_PHILOX)).set_slab(0, 7)
    assert split(10, 3) == ([4, 3, 3], [0, 4, 7])


def test_dist_slab_on_one_rank_follows_the_whole_lattice():
    """DistSlab's GPU path in a one-rank NCCL group -- the slab is the whole
    lattice with its own boundaries as halos: with the overlapped phases
    (boundary slices, pack, interior on the slab's stream while the swap
    runs on a second stream, unpack) and without, both bit-identical to the
    whole lattice"""
    import socket

    import torch
    import torch.distributed as dist
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        cfg = Q.default_config(group=3, size=(6, 4, 4, 4), precision=0, start=Q.START_HOT, prng=Q.PRNG_PHILOX,
                               beta=5.9, n_or=1, reunit_every=2, reunit_fp64=1, randseries=9)
        G = Q.Lattice(cfg)
        G.seed()
        G.init(Q.START_HOT)
        G.sweep(3)
        ns = 4 * 4 * 4
        g = G.download().reshape(12, -1, 4)
        start = Q.Lattice(cfg)
        start.seed()
        start.init(Q.START_HOT)
        for overlap in (True, False):
            D = DistSlab(cfg, dist, torch.device("cuda", 0), overlap=overlap)
            D.slab.L.seed()
            D.slab.L.upload(_to_slab(start.download(), cfg, D.slab.w, D.slab.x0, D.slab.cfg))
            D.sweep(3)
            t = D.slab.L.download().reshape(12, -1, 4)
            assert np.array_equal(t[:, ns:7 * ns, :], g[:, :6 * ns, :]), overlap
            D.slab.close()
        start.close()
        G.close()
    finally:
        dist.destroy_process_group()


def test_a_slab_phase_writes_only_its_interior_links():
    """write-set of one slab phase: the links of its direction and global
    parity in slices 1..w, never the halo slices"""
    cfg = Q.default_config(group=3, size=(8, 4, 4, 6), precision=0, start=Q.START_HOT, prng=Q.PRNG_PHILOX,
                           beta=5.8, randseries=3)
    G = Q.Lattice(cfg)
    G.seed()
    G.init(Q.START_HOT)
    table = G.download()
    w, x0 = 3, 5                                         # slices 5, 6, 7; halos 4 and 0
    S = _Slab(cfg, w, x0)
    S.L.seed()
    S.L.upload(_to_slab(table, cfg, w, x0, S.cfg))
    ns = 4 * 4 * 6
    Vs = (w + 2) * ns
    gl = np.arange(Vs)
    y, z, t, xl = gl % 4, (gl // 4) % 4, (gl // 16) % 6, gl // ns
    gpar = (xl + x0 - 1 + y + z + t) & 1                 # global parity of each slab site
    for kind in (Q.HEATBATH, Q.OVERRELAX):
        for p in (0, 1):
            for mu in range(4):
                before = S.L.download().reshape(12, -1, 4)
                for part in (0, 1):
                    S.L.slab_phase(p, mu, kind, part)
                after = S.L.download().reshape(12, -1, 4)
                for nu in range(4):
                    planes = [nu + 4 * k for k in range(3)]
                    ch = np.any(after[planes, :Vs, :] != before[planes, :Vs, :], axis=(0, 2))
                    want = (gpar == p) & (xl >= 1) & (xl <= w) & (nu == mu)
                    assert not np.any(ch & ~want), (kind, p, mu, nu)
                    if nu == mu:
                        assert ch[want].mean() > 0.99, (kind, p, mu)
    S.close()
    G.close()
