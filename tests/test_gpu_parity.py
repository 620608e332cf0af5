"""CUDA sweep vs the CPU oracle, through the C-ABI (libqg_sun.so).

Tolerances (the parity targets): link fields after phases/sweeps fed the same PRN
stream: max|dU| <= 1e-12 (FP64 links) / 2e-6 (FP32 links); plaquette and
Polyakov sums on fixed configurations: 1e-13 / 1e-6 relative; RANLUX and
Philox streams: bit-exact.
"""
import ctypes

import numpy as np
import pytest

import _oracle as O
import qcdgpu_b200 as Q

pytestmark = pytest.mark.gpu

TOL_U = {0: 2e-6, 1: 1e-12}
INSTANCES = 512


def make_pair(group, dims, precision, start=Q.START_COLD, prng=Q.PRNG_RANLUX, beta=6.0, nhit=10, nskip=223,
              n_or=0, reunit_every=1, reunit_fp64=0, phi=0.0, omega=0.0):
    L = Q.Lattice(Q.default_config(group=group, size=dims, precision=precision, start=start, prng=prng, beta=beta,
                                   nhit=nhit, ranlux_nskip=nskip, prng_instances=INSTANCES, randseries=54,
                                   row_align=64, n_or=n_or, reunit_every=reunit_every, reunit_fp64=reunit_fp64,
                                   phi=phi, omega=omega))
    c = O.make_cfg(group=group, dims=dims, precision=precision, beta=beta, nhit=nhit, row_align=64,
                   gid_mode=(start == Q.START_GID), phi=phi, omega=omega)
    return L, c


def maxdiff(a, b):
    return float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64))))


def cold_table(c):
    t = O.new_table(c)
    O.lib.ol_init_cold(ctypes.byref(c), O.vp(t))
    return t


# ------------------------------------------------------------------ PRNG
@pytest.mark.parametrize("nskip", [223, 389, 97, 48, 24])
def test_ranlux_batches_bit_exact(nskip):
    L, c = make_pair(3, (4, 4, 4, 4), 0, nskip=nskip)
    info = L.info()
    R = O.Ranlux(54, INSTANCES, nskip)
    L.seed(54)                                   # PRNG::initialize: one produce()
    for k in range(4):
        if k:
            L.produce()
        ref = R.batch(info.prng_samples)
        got = L.prns_download()
        assert got.view(np.uint32).tolist() == ref.view(np.uint32).tolist(), "batch %d" % k
    assert L.info().prng_counter == 4


def test_ranlux_default_instances_bit_exact():
    L = Q.Lattice(Q.default_config(group=3, size=(4, 4, 4, 4), precision=0, start=Q.START_COLD))
    info = L.info()
    R = O.Ranlux(54, 16384, 223)
    L.seed(54)
    L.produce()
    R.batch(info.prng_samples)
    assert np.array_equal(L.prns_download().view(np.uint32), R.batch(info.prng_samples).view(np.uint32))


def split_parts(instances, samples):
    """the number of threads per generator the library splits a batch over
    (ranlux_split_parts in qg_ranlux.cu)"""
    if samples % 6:
        return 1
    parts = min((1 << 17) // instances, samples // 6 // 8, 16)
    return parts if parts >= 2 else 1


@pytest.mark.parametrize("dims,instances,nskip,batches", [((8, 8, 8, 8), 512, 389, 3), ((8, 8, 8, 8), 256, 24, 3),
                                                          ((16, 16, 16, 16), 2048, 223, 3),
                                                          ((32, 32, 32, 32), 16384, 223, 1)])
def test_ranlux_split_batches_bit_exact(dims, instances, nskip, batches):
    """Batches of whole 24-output luxury blocks are produced with each
    generator's batch split over several threads, every segment started
    from the batch-start state jumped ahead modulo 2^576 - 2^240 + 1: the
    batches equal the oracle's serial stream bit for bit, batch after
    batch (the last case is the bench workload's generator, 16384
    instances at 32^4)"""
    L = Q.Lattice(Q.default_config(group=3, size=dims, precision=0, start=Q.START_COLD, prng=Q.PRNG_RANLUX,
                                   ranlux_nskip=nskip, prng_instances=instances, randseries=54, row_align=64))
    S = L.info().prng_samples
    assert split_parts(instances, S) > 1, S
    R = O.Ranlux(54, instances, nskip)
    L.seed(54)
    for k in range(batches):
        if k:
            L.produce()
        assert np.array_equal(L.prns_download().view(np.uint32), R.batch(S).view(np.uint32)), k
    L.close()


# ------------------------------------------------------- layout / starts
@pytest.mark.parametrize("group,precision", [(3, 0), (3, 1), (2, 0), (2, 1)])
def test_layout_roundtrip(group, precision):
    L, c = make_pair(group, (4, 6, 2, 8), precision)
    rng = np.random.default_rng(1)
    a = rng.standard_normal(L.info().ref_elems).astype(np.float64 if precision else np.float32)
    V = O.volume(c)
    for p in range(12 if group == 3 else 4):       # padding rows are not stored
        a[(p * c.rowsize + V) * 4:(p + 1) * c.rowsize * 4] = 0
    L.upload(a)
    assert np.array_equal(L.download(), a)


@pytest.mark.parametrize("group,precision", [(3, 0), (3, 1), (2, 0), (2, 1)])
def test_gid_and_cold_starts(group, precision):
    for start, init in ((Q.START_GID, O.lib.ol_init_gid), (Q.START_COLD, O.lib.ol_init_cold)):
        L, c = make_pair(group, (4, 4, 6, 4), precision, start=start)
        L.init(start)
        t = O.new_table(c)
        init(ctypes.byref(c), O.vp(t))
        assert maxdiff(L.download(), t) <= TOL_U[precision]


@pytest.mark.parametrize("group,precision", [(3, 0), (3, 1), (2, 0), (2, 1)])
def test_hot_start_ranlux(group, precision):
    L, c = make_pair(group, (4, 4, 4, 4), precision, start=Q.START_HOT)
    info = L.info()
    R = O.Ranlux(54, INSTANCES)
    L.seed(54)
    L.init(Q.START_HOT)
    R.batch(info.prng_samples)
    t = O.new_table(c)
    for mu in range(4):
        O.lib.ol_init_hot_dir(ctypes.byref(c), O.vp(t), mu, O.vp(R.batch(info.prng_samples)))
    assert maxdiff(L.download(), t) <= TOL_U[precision] * 4


# ------------------------------------------------------------- updates
def oracle_sweep_ranlux(c, t, R, samples):
    for par in (1, 0):
        for mu in range(4):
            O.phase_hb(c, t, par, mu, prns=R.batch(samples))


@pytest.mark.parametrize("group,precision,dims", [(3, 1, (4, 4, 4, 4)), (3, 0, (4, 4, 4, 4)),
                                                  (2, 1, (4, 6, 2, 4)), (2, 0, (4, 6, 2, 4)),
                                                  (3, 1, (2, 4, 6, 4))])
def test_heatbath_phases_ranlux(group, precision, dims):
    """Each update_{odd,even}_{X..T} fed the same RANLUX batch as the oracle."""
    L, c = make_pair(group, dims, precision, start=Q.START_HOT, beta=5.7 if group == 3 else 2.3)
    info = L.info()
    R = O.Ranlux(54, INSTANCES)
    L.seed(54)
    L.init(Q.START_HOT)
    R.batch(info.prng_samples)
    t = O.new_table(c)
    for mu in range(4):
        O.lib.ol_init_hot_dir(ctypes.byref(c), O.vp(t), mu, O.vp(R.batch(info.prng_samples)))
    L.upload(t)                                  # start both from the oracle's table
    for par in (1, 0):
        for mu in range(4):
            L.produce()
            L.phase(par, mu)
            O.phase_hb(c, t, par, mu, prns=R.batch(info.prng_samples))
            d = maxdiff(L.download(), t)
            assert d <= TOL_U[precision], (par, mu, d)


@pytest.mark.parametrize("group,precision", [(3, 1), (3, 0), (2, 1), (2, 0)])
def test_sweeps_ranlux_reference_cadence(group, precision):
    """qg_sweep = lattice_simulate's working cycle: 8 x (produce, phase), GS."""
    L, c = make_pair(group, (4, 4, 4, 4), precision, start=Q.START_COLD, beta=6.0 if group == 3 else 2.3)
    info = L.info()
    R = O.Ranlux(54, INSTANCES)
    L.seed(54)
    L.init(Q.START_COLD)
    R.batch(info.prng_samples)
    t = cold_table(c)
    for s in range(2):
        L.sweep(1)
        oracle_sweep_ranlux(c, t, R, info.prng_samples)
        O.lib.ol_gramschmidt(ctypes.byref(c), O.vp(t))
        d = maxdiff(L.download(), t)
        assert d <= TOL_U[precision] * (1 + s), (s, d)
    assert L.info().prng_counter == 1 + 16


@pytest.mark.parametrize("precision,look", [(1, 1), (0, 0)])
def test_sweeps_with_split_ranlux_batches(precision, look):
    """qg_sweep in RANLUX mode at a size whose batches are whole luxury
    blocks (8^4, 512 generators: each batch over 2 threads per generator),
    with and without the lookahead: the links follow the oracle's sweep fed
    the serial stream"""
    L, c = make_pair(3, (8, 8, 8, 8), precision, start=Q.START_COLD, beta=6.0)
    L.set_prng_lookahead(look)
    S = L.info().prng_samples
    assert split_parts(INSTANCES, S) > 1, S
    R = O.Ranlux(54, INSTANCES)
    L.seed(54)
    L.init(Q.START_COLD)
    R.batch(S)
    t = cold_table(c)
    for s in range(2):
        L.sweep(1)
        oracle_sweep_ranlux(c, t, R, S)
        O.lib.ol_gramschmidt(ctypes.byref(c), O.vp(t))
        d = maxdiff(L.download(), t)
        assert d <= TOL_U[precision] * (1 + s), (s, d)
    L.close()


def _ranlux_lookahead_chain(look, precision):
    """3 sweeps in one call, one single heatbath phase, 2 more sweeps, then
    one produce: the PRN buffer after the sweeps, the links, the buffer after
    the produce and the batch counter"""
    L, c = make_pair(3, (4, 4, 4, 4), precision, n_or=1, reunit_every=2, reunit_fp64=1)
    L.set_prng_lookahead(look)
    L.seed(54)
    L.init(Q.START_COLD)
    L.sweep(3)
    buf3 = L.prns_download()
    L.phase(1, 2, Q.HEATBATH)                    # reads the last batch consumed, produces none
    L.sweep(2)
    links = L.download()
    L.produce()
    nxt = L.prns_download()
    counter = L.info().prng_counter
    samples = L.info().prng_samples
    L.close()
    return c, samples, buf3, links, nxt, counter


@pytest.mark.parametrize("precision", [1, 0])
def test_ranlux_lookahead_keeps_the_stream(precision):
    """qg_sweep with the RANLUX lookahead (the next sweep's batches generated
    on a second stream while the current sweep runs) consumes the same
    batches in the same order as without it; after sweeps the PRN buffer
    holds the last batch consumed, a single phase reads it, and produce
    continues the stream from there -- against the oracle, and bit for bit
    against the context without the lookahead."""
    c, S, buf3, links, nxt, counter = _ranlux_lookahead_chain(1, precision)
    _, _, buf3_0, links_0, nxt_0, counter_0 = _ranlux_lookahead_chain(0, precision)
    assert np.array_equal(buf3.view(np.uint32), buf3_0.view(np.uint32))
    assert np.array_equal(links, links_0)
    assert np.array_equal(nxt.view(np.uint32), nxt_0.view(np.uint32))
    assert counter == counter_0 == 1 + 5 * 8 + 1
    R = O.Ranlux(54, INSTANCES)
    R.batch(S)
    t = cold_table(c)
    last = None
    for s in range(5):
        for par in (1, 0):
            for mu in range(4):
                last = R.batch(S)
                O.phase_hb(c, t, par, mu, prns=last)
        for par in (1, 0):
            for mu in range(4):
                O.lib.ol_phase_or(ctypes.byref(c), O.vp(t), par, mu)
        if s % 2 == 1:
            O.lib.ol_gramschmidt_fp64(ctypes.byref(c), O.vp(t))
        if s == 2:
            assert np.array_equal(buf3.view(np.uint32), last.view(np.uint32))
            O.phase_hb(c, t, 1, 2, prns=last)
    assert maxdiff(links, t) <= TOL_U[precision] * 5
    assert np.array_equal(nxt.view(np.uint32), R.batch(S).view(np.uint32))


@pytest.mark.parametrize("group,precision", [(3, 1), (3, 0), (2, 1), (2, 0)])
def test_sweeps_philox(group, precision):
    L, c = make_pair(group, (4, 4, 2, 6), precision, start=Q.START_COLD, prng=Q.PRNG_PHILOX,
                     beta=5.9 if group == 3 else 2.3)
    L.seed(54)
    L.init(Q.START_COLD)
    t = cold_table(c)
    key = (54, 0x5D3E1A27)
    ph = 0
    for s in range(2):
        L.sweep(1)
        for par in (1, 0):
            for mu in range(4):
                O.phase_hb(c, t, par, mu, philox=(key[0], key[1], ph))
                ph += 1
        O.lib.ol_gramschmidt(ctypes.byref(c), O.vp(t))
        d = maxdiff(L.download(), t)
        assert d <= TOL_U[precision] * (1 + s), (s, d)
    assert L.info().phase_counter == 16


@pytest.mark.parametrize("group,precision", [(3, 1), (3, 0), (2, 1), (2, 0)])
def test_sweeps_bit_exact(group, precision):
    """Same operation sequence on both sides (explicit fma, own sin/cos/log):
    three heatbath + overrelaxation sweeps reproduce the oracle bit for bit."""
    L, c = make_pair(group, (4, 4, 4, 4), precision, start=Q.START_COLD, prng=Q.PRNG_PHILOX,
                     beta=5.8 if group == 3 else 2.3, n_or=1, reunit_every=3, reunit_fp64=0)
    L.seed(54)
    L.init(Q.START_COLD)
    t = cold_table(c)
    ph = 0
    for s in range(3):
        L.sweep(1)
        for par in (1, 0):
            for mu in range(4):
                O.phase_hb(c, t, par, mu, philox=(54, 0x5D3E1A27, ph))
                ph += 1
        for par in (1, 0):
            for mu in range(4):
                O.lib.ol_phase_or(ctypes.byref(c), O.vp(t), par, mu)
    O.lib.ol_gramschmidt(ctypes.byref(c), O.vp(t))
    g = L.download()
    assert np.array_equal(g, t), "max|dU| = %g" % maxdiff(g, t)


@pytest.mark.parametrize("group,precision", [(3, 1), (3, 0), (2, 1), (2, 0)])
def test_overrelaxation_sweeps(group, precision):
    """1 heatbath + 2 overrelaxation sweeps, GS every 2 sweeps in FP64."""
    L, c = make_pair(group, (4, 4, 4, 4), precision, start=Q.START_COLD, prng=Q.PRNG_PHILOX,
                     beta=6.0 if group == 3 else 2.3, n_or=2, reunit_every=2, reunit_fp64=1)
    L.seed(54)
    L.init(Q.START_COLD)
    t = cold_table(c)
    ph = 0
    for s in range(4):
        L.sweep(1)
        for par in (1, 0):
            for mu in range(4):
                O.phase_hb(c, t, par, mu, philox=(54, 0x5D3E1A27, ph))
                ph += 1
        for k in range(2):
            for par in (1, 0):
                for mu in range(4):
                    O.lib.ol_phase_or(ctypes.byref(c), O.vp(t), par, mu)
        if s % 2 == 1:
            O.lib.ol_gramschmidt_fp64(ctypes.byref(c), O.vp(t))
        d = maxdiff(L.download(), t)
        assert d <= TOL_U[precision] * 4, (s, d)


@pytest.mark.parametrize("group,precision", [(3, 1), (3, 0), (2, 1), (2, 0)])
def test_gid_mode_sweeps(group, precision):
    L, c = make_pair(group, (4, 4, 4, 4), precision, start=Q.START_GID, beta=6.0)
    L.init(Q.START_GID)
    t = O.new_table(c)
    O.lib.ol_init_gid(ctypes.byref(c), O.vp(t))
    for s in range(2):
        L.sweep(1)
        for par in (1, 0):
            for mu in range(4):
                O.phase_hb(c, t, par, mu, philox=(0, 0, 0))
        O.lib.ol_gramschmidt(ctypes.byref(c), O.vp(t))
        assert maxdiff(L.download(), t) <= TOL_U[precision] * (1 + s)


def test_twisted_boundary_phase():
    L, c = make_pair(3, (4, 4, 4, 4), 1, start=Q.START_HOT, phi=0.3, omega=0.7)
    info = L.info()
    R = O.Ranlux(54, INSTANCES)
    L.seed(54)
    L.init(Q.START_HOT)
    R.batch(info.prng_samples)
    t = O.new_table(c)
    for mu in range(4):
        O.lib.ol_init_hot_dir(ctypes.byref(c), O.vp(t), mu, O.vp(R.batch(info.prng_samples)))
    for par, mu in ((1, 1), (0, 0)):
        L.produce()
        L.phase(par, mu)
        O.phase_hb(c, t, par, mu, prns=R.batch(info.prng_samples))
    assert maxdiff(L.download(), t) <= 1e-12
    a, b = L.plaquette_sums(), O.plaquette(c, t)
    assert np.allclose(a, b, rtol=1e-13, atol=0)


def test_sweep_phase_times_continue_the_sweep_chain():
    """qg_sweep_phase_times runs the qg_sweep chain: after it and further
    sweeps the links and counters equal, bit for bit, those of qg_sweep over
    the same number of sweeps (a reunitarisation falls inside the timed
    sweeps); the in-graph phase durations are positive; the RANLUX mode and
    out-of-range sweep counts are refused"""
    out = []
    for timed in (False, True):
        L = Q.Lattice(Q.default_config(group=3, size=(8, 8, 8, 8), precision=0, start=Q.START_HOT,
                                       prng=Q.PRNG_PHILOX, beta=6.0, n_or=2, reunit_every=3, reunit_fp64=1,
                                       randseries=54))
        L.seed(54)
        L.init()
        L.sweep(2)
        if timed:
            hb, orx, sw = L.sweep_phase_times(5)
            assert hb > 0 and orx > 0 and sw > 8 * hb + 16 * orx, (hb, orx, sw)
            for bad in (0, 257):
                with pytest.raises(Q.QGError):
                    L.sweep_phase_times(bad)
        else:
            L.sweep(5)
        L.sweep(2)
        info = L.info()
        out.append((L.download(), info.phase_counter, info.sweeps_done))
        L.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1:] == out[1][1:]
    L, c = make_pair(3, (4, 4, 4, 4), 0, start=Q.START_COLD, prng=Q.PRNG_RANLUX)
    L.seed(54)
    L.init(Q.START_COLD)
    with pytest.raises(Q.QGError):
        L.sweep_phase_times(2)
    L.close()


# --------------------------------------------------------- observables
def hot_config(group, dims, precision, sweeps=2):
    L, c = make_pair(group, dims, precision, start=Q.START_HOT, prng=Q.PRNG_RANLUX, beta=5.8 if group == 3 else 2.3)
    L.seed(54)
    L.init(Q.START_HOT)
    L.sweep(sweeps)
    return L, c, L.download()


@pytest.mark.parametrize("group,precision", [(3, 1), (3, 0), (2, 1), (2, 0)])
def test_plaquette_action_polyakov_wilson(group, precision):
    L, c, t = hot_config(group, (4, 6, 4, 8), precision)
    sp, tp = L.plaquette_sums()
    osp, otp = O.plaquette(c, t)
    assert abs(sp - osp) <= 1e-13 * abs(osp) and abs(tp - otp) <= 1e-13 * abs(otp)
    assert np.allclose(L.action_sums(), O.action(c, t), rtol=1e-13, atol=0)
    prel = 1e-13 if precision else 1e-6
    gp, op = L.polyakov_sums(), O.polyakov(c, t)
    scale = 4 * 6 * 4 * group
    assert all(abs(a - b) <= prel * scale for a, b in zip(gp, op)), (gp, op)
    for R, T in ((1, 1), (2, 3), (3, 2)):
        w, ow = L.wilson_sum(R, T), O.wilson(c, t, R, T)
        assert abs(w - ow) <= 1e-12 * 3 * O.volume(c) * group, (R, T, w, ow)
    # W(1,1) summed over i in {x,y,z} = temporal plaquette sum
    assert abs(L.wilson_sum(1, 1) - tp) <= 1e-12 * abs(tp)


@pytest.mark.parametrize("group,precision,twist", [(3, 0, False), (2, 0, False), (3, 0, True), (2, 0, True),
                                                   (3, 1, False)])
def test_plaquette_f32_products_match_oracle_and_fp64(group, precision, twist):
    """QG_MEAS_PLAQUETTE_F32 (each plaquette's products and trace in FP32,
    site and lattice sums in FP64): every site's six traces are the
    oracle's FP32 restatement bit for bit, so the sums agree to the FP64
    summation-order level; the normalised plaquette is within 1e-6 of the
    FP64-product plaquette (FP64 links: the same values); the queued form
    returns the same sums"""
    phi, omega = (0.3, 0.7) if twist else (0.0, 0.0)
    L, c = make_pair(group, (4, 6, 6, 8), precision, start=Q.START_HOT, prng=Q.PRNG_PHILOX,
                     beta=5.8 if group == 3 else 2.3, phi=phi, omega=omega)
    L.seed(54)
    L.init()
    L.sweep(2)
    tab = L.download()
    norm = 3 * O.volume(c) * group
    g32, o32 = L.plaquette_sums_f32(), O.plaquette_f32(c, tab)
    assert all(abs(a - b) <= 1e-13 * norm for a, b in zip(g32, o32)), (g32, o32)
    g64 = L.plaquette_sums()
    if precision:
        assert g32 == g64
    else:
        assert max(abs(a - b) for a, b in zip(g32, g64)) / norm <= 1e-6, (g32, g64)
    tk = L.measure_enqueue(Q.MEAS_PLAQUETTE_F32)
    assert L.measure_fetch(tk)[:2] == g32
    L.close()


def test_cold_observables_exact():
    for g in (2, 3):
        L, c = make_pair(g, (4, 4, 4, 6), 0)
        L.init(Q.START_COLD)
        V = O.volume(c)
        assert L.plaquette_sums() == (3.0 * V * g, 3.0 * V * g)
        assert L.polyakov_sums()[:2] == (4 * 4 * 4 * g, 0.0)
        assert L.action_sums() == (0.0, 0.0)


def test_reunitarize_parity():
    for fp64 in (0, 1):
        L, c, t = hot_config(3, (4, 4, 4, 4), 0, sweeps=1)
        rng = np.random.default_rng(3)
        t = (t + 1e-3 * rng.standard_normal(t.size)).astype(np.float32)
        L.upload(t)
        L.reunitarize(fp64=bool(fp64))
        (O.lib.ol_gramschmidt_fp64 if fp64 else O.lib.ol_gramschmidt)(ctypes.byref(c), O.vp(t))
        assert maxdiff(L.download(), t) <= 2e-7


# ----------------------------------------------------- full-size properties
@pytest.mark.parametrize("prng", [Q.PRNG_PHILOX, Q.PRNG_RANLUX])
def test_bench_config_properties(prng):
    """SU(3) 32^4 beta=6.0 FP32, HB + 4 OR: the field stays in SU(3), the
    plaquette moves from 3 toward its equilibrium, and reruns are bitwise
    reproducible."""
    res = []
    for rep in range(2):
        L = Q.Lattice(Q.default_config(group=3, size=32, precision=0, start=Q.START_COLD, prng=prng, beta=6.0,
                                       n_or=4, reunit_every=10, reunit_fp64=1, prng_instances=16384))
        L.seed(54)
        L.init(Q.START_COLD)
        L.sweep(3)
        p = L.plaquette()
        res.append((p, L.polyakov()))
        if rep == 0:
            a = L.download().reshape(12, -1, 4)[:, :32 ** 4, :].astype(np.float64)
            r1 = a[0:4, :, :3] + 1j * a[4:8, :, :3]
            n = np.sum(np.abs(r1) ** 2, axis=-1)
            assert np.max(np.abs(n - 1)) < 1e-5
        L.close()
    assert res[0] == res[1]
    sp, tp, tot = res[0][0]
    assert 1.6 < tot < 2.6


def test_tune_restores_field_and_keeps_results():
    """qg_tune times launch shapes on a copy of the state it restores; the
    shapes compute the same sequence, so tuned and untuned chains agree."""
    outs = []
    for tune in (False, True):
        L = Q.Lattice(Q.default_config(group=3, size=(8, 8, 8, 8), precision=0, start=Q.START_COLD,
                                       prng=Q.PRNG_PHILOX, beta=6.0, n_or=2, reunit_every=2))
        L.seed(54)
        L.init()
        L.sweep(1)
        before = L.download()
        if tune:
            t = L.tune(reps=2)
            assert len(t) == Q.TUNE_SHAPES and all(a > 0 and b > 0 for a, b in t)
            assert np.array_equal(L.download(), before)
            assert L.info().phase_counter == 8
        L.sweep(2)
        outs.append(L.download())
        L.close()
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("group,precision,prng", [(3, 0, Q.PRNG_PHILOX), (3, 0, Q.PRNG_RANLUX), (3, 1, Q.PRNG_PHILOX),
                                                  (2, 0, Q.PRNG_PHILOX), (2, 1, Q.PRNG_RANLUX)])
def test_every_launch_shape_gives_the_same_chain(group, precision, prng):
    """Each launch shape (registers, register caps, staple staged through
    shared memory) performs the same operation sequence: heatbath and
    overrelaxation sweeps from a hot start agree bit for bit."""
    dims = (6, 4, 4, 8) if group == 2 or precision == 1 else (3, 4, 3, 6)   # V/2 = 108 ... and odd V/4
    outs = []
    for shape in range(Q.TUNE_SHAPES):
        L = Q.Lattice(Q.default_config(group=group, size=dims, precision=precision, start=Q.START_HOT, prng=prng,
                                       beta=5.9 if group == 3 else 2.3, prng_instances=INSTANCES, randseries=54,
                                       n_or=2, reunit_every=2))
        L.set_shapes(shape, shape)
        assert L.shapes() == (shape, shape)
        L.seed(54)
        L.init()
        L.sweep(2)
        outs.append(L.download())
        L.close()
    for k in range(1, len(outs)):
        assert np.array_equal(outs[0], outs[k]), "shape %d differs from shape 0" % k


def test_set_shapes_rejects_out_of_range():
    L = Q.Lattice(Q.default_config(group=3, size=(4, 4, 4, 4), precision=0, start=Q.START_COLD))
    with pytest.raises(Q.QGError):
        L.set_shapes(Q.TUNE_SHAPES, 0)
    with pytest.raises(Q.QGError):
        L.set_shapes(0, -1)
    L.close()


@pytest.mark.parametrize("group,precision,twist", [(3, 0, False), (3, 1, False), (2, 1, False), (3, 0, True),
                                                   (2, 1, True)])
def test_wilson_all_loops_match_single_loops_and_oracle(group, precision, twist):
    """qg_measure_wilson_all (every R x T up to Rmax x Tmax in one launch)
    equals qg_measure_wilson loop by loop and the oracle's Wilson loops, to
    the FP64 summation-order level; with a twisted boundary both kernels
    take their twisted form"""
    phi, omega = (0.3, 0.7) if twist else (0.0, 0.0)
    L, c = make_pair(group, (4, 6, 6, 8), precision, start=Q.START_HOT, prng=Q.PRNG_PHILOX, beta=5.8,
                     phi=phi, omega=omega)
    L.seed(54)
    L.init()
    L.sweep(2)
    tab = L.download()
    W = L.wilson_all(4, 6)
    assert W.shape == (4, 6)
    for R in range(1, 5):
        for T in range(1, 7):
            single = L.wilson_sum(R, T)
            assert abs(W[R - 1, T - 1] - single) <= 1e-12 * abs(single) + 1e-9, (R, T)
    for R, T in ((1, 1), (2, 3), (4, 6)):
        ow = O.wilson(c, tab, R, T)
        assert abs(W[R - 1, T - 1] - ow) <= 1e-11 * abs(ow) + 1e-8, (R, T)
    if precision == 0:                                   # FP32 products, FP64 trace sums
        W32 = L.wilson_all(4, 6, fp64_products=False)
        V = 4 * 6 * 6 * 8
        assert np.max(np.abs(W32 - W)) <= 3e-6 * 3 * V
    with pytest.raises(Q.QGError):
        L.wilson_all(5, 6)
    with pytest.raises(Q.QGError):
        L.wilson_all(4, 17)
    L.close()


# ------------------------------------------------ F_munu and profiles
@pytest.mark.parametrize("group,precision,twist", [(3, 1, False), (3, 0, False), (2, 1, False), (2, 0, False),
                                                   (3, 1, True)])
def test_fmunu_and_profiles_match_oracle(group, precision, twist):
    """qg_measure_fmunu and the action / Polyakov profiles equal the oracle
    on a thermalising configuration (FP64 sums; tolerances of the plaquette
    and Polyakov parity), every generator pair and both fields"""
    phi, omega = (0.3, 0.7) if twist else (0.0, 0.0)
    dims = (6, 4, 4, 8)
    L, c = make_pair(group, dims, precision, start=Q.START_HOT, prng=Q.PRNG_RANLUX,
                     beta=5.8 if group == 3 else 2.3, phi=phi, omega=omega)
    L.seed(54)
    L.init(Q.START_HOT)
    L.sweep(2)
    t = L.download()
    V = O.volume(c)
    pairs = [(1, 5), (2, 6), (3, 8), (4, 7)] if group == 3 else [(3, 2), (1, 2)]
    for field in (Q.FMUNU_H, Q.FMUNU_E):
        for i1, i2 in pairs:
            g, o = L.fmunu(field, i1, i2), O.fmunu(c, t, field, i1, i2)
            assert np.max(np.abs(g - o)) <= 1e-12 * V, (field, i1, i2, g, o)
            assert np.any(o != 0)
    sp = L.action_sums()
    for axis in range(3):
        a, oa = L.action_profile(axis), O.action_profile(c, t, axis)
        assert a.shape == (dims[axis], 2)
        assert np.allclose(a, oa, rtol=1e-12, atol=1e-12 * V), axis
        assert abs(a[:, 0].sum() - sp[0]) <= 1e-12 * abs(sp[0])
        p, op = L.polyakov_profile(axis), O.polyakov_profile(c, t, axis)
        prel = 1e-12 if precision else 1e-6
        assert np.max(np.abs(p - op)) <= prel * V / dims[3] * group, axis
    with pytest.raises(Q.QGError):
        L.fmunu(2, 3, 8)
    with pytest.raises(Q.QGError):
        L.fmunu(0, 0, 8)
    with pytest.raises(Q.QGError):
        L.action_profile(3)
    L.close()


def test_fmunu_and_profiles_cold():
    """cold start: F = 0 exactly, flat profiles (action 0, Polyakov N per site)"""
    for g in (2, 3):
        dims = (4, 6, 4, 6)
        L, c = make_pair(g, dims, 0)
        L.init(Q.START_COLD)
        assert np.all(L.fmunu(Q.FMUNU_H) == 0.0) and np.all(L.fmunu(Q.FMUNU_E) == 0.0)
        for axis in range(3):
            assert np.all(L.action_profile(axis) == 0.0)
            p = L.polyakov_profile(axis)
            per = dims[0] * dims[1] * dims[2] // dims[axis]
            assert np.all(p[:, 0] == g * per) and np.all(p[:, 1] == 0.0)
        L.close()


def test_async_measurements_and_parameter_staging():
    """qg_measure_enqueue / _fetch give qg_measure's values; parameter
    uploads queued back to back (no stream wait) apply in stream order; old
    or unknown tickets are errors"""
    L, c, t = hot_config(3, (4, 6, 4, 8), 1)
    sp, tp = L.plaquette_sums()
    assert L.measure_fetch(L.measure_enqueue(Q.MEAS_PLAQUETTE))[:2] == (sp, tp)
    assert L.measure_fetch(L.measure_enqueue(Q.MEAS_POLYAKOV)) == tuple(L.polyakov_sums())
    with pytest.raises(Q.QGError):                    # WILSONR = 7 > N1 = 4, as qg_measure_wilson
        L.measure_enqueue(Q.MEAS_WILSON)
    with pytest.raises(Q.QGError):
        L.wilson_sum()
    assert L.measure_fetch(L.measure_enqueue(Q.MEAS_ACTION))[:2] == tuple(L.action_sums())
    betas = [5.0 + 0.1 * k for k in range(20)]
    tickets = []
    for b in betas:                                   # 20 uploads, more than the 8 staging slots
        L.set_params(b)
        tickets.append(L.measure_enqueue(Q.MEAS_ACTION))
    V = O.volume(c)
    for b, tk in zip(betas, tickets):
        a = L.measure_fetch(tk)[:2]
        assert abs(a[0] - b / 3 * (9 * V - sp)) <= 1e-12 * abs(a[0])
        assert abs(a[1] - b / 3 * (9 * V - tp)) <= 1e-12 * abs(a[1])
    first = L.measure_enqueue(Q.MEAS_PLAQUETTE)
    for _ in range(Q.MEASURE_SLOTS):
        L.measure_enqueue(Q.MEAS_PLAQUETTE)
    with pytest.raises(Q.QGError):
        L.measure_fetch(first)                        # its slot was reused
    with pytest.raises(Q.QGError):
        L.measure_fetch(10 ** 9)
    L.close()


@pytest.mark.parametrize("group,precision,twist", [(3, 0, False), (3, 1, True), (2, 1, False)])
def test_one_pass_measurements_equal_the_separate_ones(group, precision, twist):
    """qg_measure_plaquette_all / _polyakov_all: totals and all three
    profiles bit-identical to qg_measure and qg_measure_*_profile"""
    phi, omega = (0.3, 0.7) if twist else (0.0, 0.0)
    L, c = make_pair(group, (6, 4, 4, 8), precision, start=Q.START_HOT, prng=Q.PRNG_RANLUX,
                     beta=5.8 if group == 3 else 2.3, phi=phi, omega=omega)
    L.seed(54)
    L.init(Q.START_HOT)
    L.sweep(1)
    tot, prof = L.measure_all()
    assert tot[:2] == tuple(L.plaquette_sums()) and tot[2:] == tuple(L.action_sums())
    for a in range(3):
        assert np.array_equal(prof[a], L.action_profile(a)), a
    tot, prof = L.measure_all(polyakov=True)
    assert tot == tuple(L.polyakov_sums())
    for a in range(3):
        assert np.array_equal(prof[a], L.polyakov_profile(a)), a
    L.close()


# ------------------------------------------------------ write sets
def _changed_links(before, after, c, planes_per_dir):
    """gid x direction mask of links whose stored reals changed"""
    P = 12 if c.group == 3 else 4
    rows = before.size // (P * 4)
    b = before.reshape(P, rows, 4)
    a = after.reshape(P, rows, 4)
    V = int(np.prod(list(c.n)))
    out = np.zeros((V, 4), dtype=bool)
    for mu in range(4):
        planes = [mu + 4 * k for k in range(planes_per_dir)]
        out[:, mu] = np.any(a[planes, :V, :] != b[planes, :V, :], axis=(0, 2))
    return out


def _parity(c):
    n = list(c.n)
    g = np.arange(int(np.prod(n)))
    y = g % n[1]
    z = (g // n[1]) % n[2]
    t = (g // (n[1] * n[2])) % n[3]
    x = g // (n[1] * n[2] * n[3])
    return (x + y + z + t) & 1


@pytest.mark.parametrize("group,precision,shape", [(3, 0, 0), (3, 0, 4), (3, 0, 5), (3, 1, 0), (2, 0, 1), (2, 1, 0)])
def test_each_phase_writes_exactly_its_links(group, precision, shape):
    """write-set disjointness: one (parity, direction) phase of either kind
    changes the V/2 links of that parity and direction and nothing else"""
    L, c = make_pair(group, (4, 6, 4, 6), precision, start=Q.START_HOT, prng=Q.PRNG_PHILOX,
                     beta=5.8 if group == 3 else 2.3)
    L.set_shapes(shape, shape)
    L.seed(54)
    L.init(Q.START_HOT)
    par = _parity(c)
    for kind in (Q.HEATBATH, Q.OVERRELAX):
        for p in (0, 1):
            for mu in range(4):
                before = L.download()
                L.phase(p, mu, kind)
                ch = _changed_links(before, L.download(), c, 3 if group == 3 else 1)
                want = np.zeros_like(ch)
                want[:, mu] = par == p
                assert not np.any(ch & ~want), (kind, p, mu)            # nothing outside the phase's links
                assert ch[want].mean() > 0.99, (kind, p, mu)             # and (almost) all of them updated
    L.close()


@pytest.mark.parametrize("dims", [(2, 2, 2, 2), (2, 4, 2, 6), (4, 2, 6, 2), (2, 6, 4, 2)])
@pytest.mark.parametrize("group,shape", [(3, 0), (3, 3), (3, 4), (2, 0)])
def test_extents_of_two_every_shape_bit_exact(dims, group, shape):
    """Extents of 2, where a link's +1 and -1 neighbours along that
    direction are the same site (N2 = 2: one y pair per checkerboard row):
    two heatbath + overrelaxation sweeps of the register form (shape 0) and
    the staged forms (3, 4) reproduce the oracle bit for bit (FP32, Philox)"""
    L, c = make_pair(group, dims, 0, start=Q.START_COLD, prng=Q.PRNG_PHILOX,
                     beta=5.8 if group == 3 else 2.3, n_or=1, reunit_every=3)
    L.set_shapes(shape, shape)
    L.seed(54)
    L.init(Q.START_COLD)
    t = cold_table(c)
    ph = 0
    for s in range(2):
        L.sweep(1)
        for par in (1, 0):
            for mu in range(4):
                O.phase_hb(c, t, par, mu, philox=(54, 0x5D3E1A27, ph))
                ph += 1
        for par in (1, 0):
            for mu in range(4):
                O.lib.ol_phase_or(ctypes.byref(c), O.vp(t), par, mu)
    g = L.download()
    assert np.array_equal(g, t), "max|dU| = %g" % maxdiff(g, t)
