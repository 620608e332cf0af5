"""Size-independent properties at the run configurations' full sizes (the
oracle checks the same code paths bit for bit on small lattices):

* SU(3) 64^4 beta=6.2 FP32, HB + 4 OR (3.2 GB of links): reruns from the
  same seed are bitwise reproducible, the one-pass measurements equal the
  separate ones, all R x T <= 8 x 8 Wilson loops with FP32 products agree
  with the FP64-product kernel to FP32 accuracy, so does the FP32-product
  plaquette (within 1e-6), and W(1,1) equals the temporal plaquette sum (SU(3) rows are checked at 32^4, in
  test_gpu_parity.py, where the field fits a host download comfortably).
* SU(3) 32^4 beta=6.0 FP32 in the reference's RANLUX mode (16384
  instances, 277 MB per batch): the lookahead sweep (next sweep's batches
  generated alongside) leaves the links and the PRN buffer bit-identical to
  the plain sweep.
* SU(3) 24^3 x 6 beta=5.9 cold start: FP32 links and the all-FP64 run, fed
  the same Philox stream, agree after one sweep to FP32 accuracy.
"""
import numpy as np
import pytest

import qcdgpu_b200 as Q

pytestmark = pytest.mark.gpu


def test_64x4_reproducible_and_measurements_consistent():
    sums = []
    for rep in range(2):
        L = Q.Lattice(Q.default_config(group=3, size=64, precision=0, start=Q.START_COLD, prng=Q.PRNG_PHILOX,
                                       beta=6.2, n_or=4, reunit_every=10, reunit_fp64=1))
        L.seed(54)
        L.init(Q.START_COLD)
        L.sweep(2)
        plq, act, pol = L.plaquette_sums(), L.action_sums(), L.polyakov_sums()
        sums.append((tuple(plq), tuple(act), tuple(pol)))
        if rep == 0:
            tot, prof = L.measure_all()
            assert tot[:2] == tuple(plq) and tot[2:] == tuple(act)
            for a in range(3):
                assert np.array_equal(prof[a], L.action_profile(a)), a
                assert abs(prof[a][:, 0].sum() - act[0]) <= 1e-9 * abs(act[0])
            tot, prof = L.measure_all(polyakov=True)
            assert tot == tuple(pol)
            w32 = L.wilson_all(8, 8, fp64_products=False)
            w64 = L.wilson_all(8, 8, fp64_products=True)
            V = 64 ** 4
            # W(1,1) summed over the three spatial directions = the temporal plaquette sum
            assert abs(w64[0, 0] - plq[1]) <= 1e-9 * abs(plq[1])
            assert np.max(np.abs(w32 - w64)) / (3 * 3 * V) < 1e-5
            # FP32-product plaquette: within 1e-6 of the FP64-product one, normalised
            p32 = L.plaquette_sums_f32()
            assert max(abs(a - b) for a, b in zip(p32, plq)) / (3 * 3 * V) < 1e-6, (p32, plq)
        L.close()
    assert sums[0] == sums[1]
    p = (sums[0][0][0] + sums[0][0][1]) / (6 * 64 ** 4)
    assert 1.8 < p < 3.0            # two sweeps from cold: still above the beta=6.2 equilibrium (~1.85)


def test_32x4_ranlux_lookahead_equals_plain_sweep():
    out = []
    for look in (1, 0):
        L = Q.Lattice(Q.default_config(group=3, size=32, precision=0, start=Q.START_COLD, prng=Q.PRNG_RANLUX,
                                       beta=6.0, n_or=4, reunit_every=10, reunit_fp64=1, prng_instances=16384))
        L.set_prng_lookahead(look)
        L.seed(54)
        L.init(Q.START_COLD)
        L.sweep(2)
        out.append((L.download(), L.prns_download(), L.info().prng_counter))
        L.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1].view(np.uint32), out[1][1].view(np.uint32))
    assert out[0][2] == out[1][2] == 1 + 16


def test_24x6_fp32_follows_fp64_for_one_sweep():
    res = []
    for precision in (0, 1):
        L = Q.Lattice(Q.default_config(group=3, size=(24, 24, 24, 6), precision=precision, start=Q.START_COLD,
                                       prng=Q.PRNG_PHILOX, beta=5.9, n_or=4, reunit_every=10, reunit_fp64=1))
        L.seed(54)
        L.init(Q.START_COLD)
        L.sweep(1)
        res.append((L.download().astype(np.float64), L.plaquette()[2]))
        L.close()
    d = np.max(np.abs(res[0][0] - res[1][0]))
    assert d < 1e-4, d
    assert abs(res[0][1] - res[1][1]) < 1e-5


def test_lattice_beyond_device_memory_fails_cleanly():
    """A valid lattice whose links exceed the device memory (160^3 x 256
    SU(3) FP32: 1.05e9 sites, 201 GB of links against 180 GB of HBM) is
    refused by qg_create with a CUDA allocation error, not a crash, and
    the process goes on creating and sweeping lattices"""
    with pytest.raises(Q.QGError) as e:
        Q.Lattice(Q.default_config(group=3, size=(160, 160, 160, 256), precision=0, start=Q.START_COLD,
                                   prng=Q.PRNG_PHILOX))
    assert "memory" in str(e.value).lower() or "alloc" in str(e.value).lower(), str(e.value)
    L = Q.Lattice(Q.default_config(group=3, size=(8, 8, 8, 8), precision=0, start=Q.START_COLD,
                                   prng=Q.PRNG_PHILOX, n_or=1))
    L.seed(54)
    L.init()
    L.sweep(2)
    sp, tp = L.plaquette_sums()
    assert 0 < sp < 3 * 8 ** 4 * 3 and 0 < tp < 3 * 8 ** 4 * 3
    L.close()
