"""Batched ensembles (qg_batch) against single contexts: every ensemble of
a heterogeneous batch -- different extents, couplings and seeds, one launch
per phase over all of them -- follows the chain a single context with its
settings follows, bit for bit, and the device-resident measurement series
equals the single context's qg_measure sums at the same sweeps."""
import numpy as np
import pytest

import qcdgpu_b200 as Q

pytestmark = pytest.mark.gpu

ENSEMBLES = [((4, 4, 4, 4), 5.5, 101), ((6, 4, 4, 8), 5.8, 102), ((4, 6, 6, 4), 6.0, 103),
             ((8, 8, 8, 4), 6.2, 104), ((4, 4, 8, 6), 5.9, 105)]


def common(group, precision, **kw):
    return Q.default_config(group=group, precision=precision, prng=Q.PRNG_PHILOX, n_or=2, reunit_every=3,
                            reunit_fp64=1, nhit=10, row_align=64, **kw)


@pytest.mark.parametrize("group,precision,shape,start", [(3, 0, 4, Q.START_HOT), (3, 0, 0, Q.START_COLD),
                                                         (3, 1, 0, Q.START_HAAR), (2, 1, 0, Q.START_HOT),
                                                         (2, 0, 4, Q.START_COLD)])
def test_batch_equals_single_contexts(group, precision, shape, start):
    sweeps, every = 7, 2
    B = Q.Batch(common(group, precision), ENSEMBLES, max_measurements=8)
    B.set_shape(shape)
    B.init(start)
    B.run(sweeps, measure_every=every)
    ser = B.series()
    assert ser.shape == (sweeps // every, len(ENSEMBLES), 8)
    info = B.info()
    assert info["sweeps"] == sweeps and info["sites"] == sum(int(np.prod(s)) for s, _, _ in ENSEMBLES)
    for e, (size, beta, series) in enumerate(ENSEMBLES):
        L = Q.Lattice(common(group, precision, size=size, beta=beta, randseries=series, start=start))
        L.seed(series)
        L.init(start)
        m = 0
        for k in range(1, sweeps + 1):
            L.sweep(1)
            if k % every == 0:
                got = np.concatenate([L.plaquette_sums(), L.action_sums(), L.polyakov_sums()])
                assert np.array_equal(got, ser[m, e]), (e, k, got, ser[m, e])
                m += 1
        assert np.array_equal(L.download(), B.download(e)), e
        L.close()
    B.close()


@pytest.mark.parametrize("group", [3, 2])
def test_batch_fp32_product_measurements_equal_single_contexts(group):
    """qg_batch_set_measure_products(1): the series' plaquette sums are the
    single context's QG_MEAS_PLAQUETTE_F32 sums bit for bit, the Polyakov
    sums are unchanged, the action follows the FP64-product action to FP32
    accuracy; switching back gives the FP64-product sums again"""
    sweeps, every = 4, 2
    B = Q.Batch(common(group, 0), ENSEMBLES, max_measurements=4)
    B.init(Q.START_HOT)
    B.set_measure_products(True)
    B.run(sweeps, measure_every=every)
    B.set_measure_products(False)
    B.run(2, measure_every=2)
    ser = B.series()
    assert ser.shape == (3, len(ENSEMBLES), 8)
    for e, (size, beta, series) in enumerate(ENSEMBLES):
        L = Q.Lattice(common(group, 0, size=size, beta=beta, randseries=series, start=Q.START_HOT))
        L.seed(series)
        L.init(Q.START_HOT)
        norm = 3 * int(np.prod(size)) * group
        for m, k in enumerate((2, 4, 6)):
            L.sweep(2)
            if k < 6:
                assert np.array_equal(np.array(L.plaquette_sums_f32()), ser[m, e, :2]), (e, k)
                assert np.max(np.abs(np.array(L.action_sums()) - ser[m, e, 2:4])) <= 1e-6 * beta / group * norm
            else:
                assert np.array_equal(np.array(L.plaquette_sums()), ser[m, e, :2]), (e, k)
                assert np.array_equal(np.array(L.action_sums()), ser[m, e, 2:4]), (e, k)
            assert np.array_equal(np.array(L.polyakov_sums()), ser[m, e, 4:]), (e, k)
        L.close()
    B.close()


def test_batch_fp32_product_flag_leaves_fp64_batches_unchanged():
    """FP64-link batches measure with FP64 products whatever the flag"""
    outs = []
    for flag in (False, True):
        B = Q.Batch(common(3, 1), ENSEMBLES[:2], max_measurements=2)
        B.init(Q.START_HOT)
        B.set_measure_products(flag)
        B.run(2, measure_every=1)
        outs.append(B.series())
        B.close()
    assert np.array_equal(outs[0], outs[1])


def test_every_batch_shape_and_the_tuner_give_the_same_chain():
    """the batched launch shapes 0-4 compute the same operation sequence,
    and qg_batch_tune restores the fields it times on: all runs end with the
    same links and series, bit for bit"""
    def run(shapes=None, tune=False):
        B = Q.Batch(common(3, 0), ENSEMBLES, max_measurements=4)
        B.init(Q.START_HOT)
        B.run(2, measure_every=1)
        if tune:
            t = B.tune(reps=2)
            assert len(t) == Q.BATCH_SHAPES and all(a > 0 and b > 0 for a, b in t)
            assert all(0 <= s < Q.BATCH_SHAPES for s in B.shapes())
        else:
            B.set_shapes(*shapes)
            assert B.shapes() == shapes
        B.run(2, measure_every=1)
        out = (B.series(), [B.download(e) for e in range(len(ENSEMBLES))])
        B.close()
        return out
    ref_ser, ref_links = run((0, 0))
    for shapes in [(1, 2), (2, 1), (3, 4), (4, 3), (4, 4)]:
        ser, links = run(shapes)
        assert np.array_equal(ser, ref_ser), shapes
        assert all(np.array_equal(a, b) for a, b in zip(links, ref_links)), shapes
    ser, links = run(tune=True)
    assert np.array_equal(ser, ref_ser)
    assert all(np.array_equal(a, b) for a, b in zip(links, ref_links))
    B = Q.Batch(common(3, 0), ENSEMBLES[:1])
    with pytest.raises(Q.QGError):
        B.set_shapes(Q.BATCH_SHAPES, 0)
    with pytest.raises(Q.QGError):
        B.set_shape(-1)
    B.close()


def test_batch_series_capacity_and_argument_checks():
    B = Q.Batch(common(3, 0), ENSEMBLES[:2], max_measurements=1)
    B.init(Q.START_COLD)
    B.run(3, measure_every=1)
    with pytest.raises(Q.QGError):
        B.series()
    B.close()
    with pytest.raises(Q.QGError):
        Q.Batch(Q.default_config(group=3, precision=0, prng=Q.PRNG_RANLUX), ENSEMBLES[:1])
    with pytest.raises(Q.QGError):
        Q.Batch(common(3, 0), [((4, 5, 4, 4), 6.0, 1)])
    with pytest.raises(Q.QGError):
        Q.Batch(common(3, 0), [((4, 4, 4, 4), 6.0, 0)])


def test_beta_scan_split_over_ranks_gives_the_same_ensembles():
    """the multi-GPU replica scheduler's shares, run here one after the
    other on one GPU, reproduce the single-batch run ensemble by ensemble
    bit for bit (each chain depends only on its RANDSERIES and the sweep
    count, not on the batch it runs in)"""
    from types import SimpleNamespace

    from qcdgpu_b200 import betascan as BS
    ens = [((8, 8, 8, 4), 5.6, 1000), ((6, 6, 6, 4), 5.8, 1001), ((8, 8, 8, 6), 6.0, 1002),
           ((4, 4, 4, 4), 5.5, 1003), ((6, 6, 6, 6), 5.9, 1004)]
    a = SimpleNamespace(n_or=2, sweeps=6, warmup=3, measure_every=1, shape=4, barrier=None)
    whole = BS.run_share(ens, list(range(len(ens))), a)
    shares = BS.partition(ens, 2, a.n_or)
    assert all(shares)
    job = BS.merge([BS.run_share(ens, s, a) for s in shares], len(ens))
    assert job["plaquette"] == whole["plaquette"]
    assert job["polyakov_abs"] == whole["polyakov_abs"]
    assert job["updates"] == whole["updates"] and job["sites"] == whole["sites"]


@pytest.mark.parametrize("group,precision,shape", [(3, 0, 4), (3, 0, 3), (3, 1, 0), (2, 0, 1)])
def test_persistent_half_sweeps_give_the_same_chain(group, precision, shape):
    """one persistent launch per half-sweep (four directions, grid barriers
    between them) gives, bit for bit, the links and series of the per-phase
    launches, heatbath and overrelaxation, with the reunitarisation and
    measurement cadences of the graph"""
    def run(persistent):
        B = Q.Batch(common(group, precision), ENSEMBLES, max_measurements=8)
        B.set_shape(shape)
        B.set_persistent(persistent)
        B.init(Q.START_HOT)
        B.run(5, measure_every=2)
        out = (B.series(), [B.download(e) for e in range(len(ENSEMBLES))])
        B.close()
        return out
    ser0, links0 = run(False)
    ser1, links1 = run(True)
    assert np.array_equal(ser0, ser1)
    assert all(np.array_equal(a, b) for a, b in zip(links0, links1))


def test_persistent_grid_barrier_times_out_and_the_batch_recovers():
    """the bounded grid barrier: one block leaves out its arrival, every
    other block's wait runs out after a second, the call reports it, and
    the batch is usable again (a fresh init and run reproduce a fresh
    batch)"""
    B = Q.Batch(common(3, 0), ENSEMBLES, max_measurements=4)
    B.set_persistent(True)
    B.init(Q.START_HOT)
    rc, msg = B.barrier_test(3)
    assert rc == Q.QG_ERR_CUDA and "grid barrier" in msg, (rc, msg)
    B.sync()                                            # the flag was cleared by the report
    B.init(Q.START_HOT)
    B.run(2, measure_every=1)
    ser = B.series()
    R = Q.Batch(common(3, 0), ENSEMBLES, max_measurements=4)
    R.init(Q.START_HOT)
    R.run(2, measure_every=1)
    assert np.array_equal(ser, R.series())
    B.close()
    R.close()
