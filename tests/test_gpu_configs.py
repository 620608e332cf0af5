"""CUDA path vs the CPU oracle at the run configurations' own lattice sizes.

The small-lattice parity tests (test_gpu_parity.py) cover every kernel form
on 2..6-site edges; these run the same comparisons on the lattices the run
configurations name, with their couplings, precisions and update mix:

  SU(2) 8^4 beta=2.3 FP64, hot start, sweep = 1 heatbath + 2 overrelaxation
  SU(3) 24^3 x 6 beta=5.9 FP32, cold start, 1 heatbath + 4 overrelaxation
  SU(3) 32^4 beta=6.0 FP32, the benchmark's lattice, launch shapes as the
        tuner picks them (and every other shape for one phase of each kind)
  SU(3) 16^4 beta=5.7 FP32, learned-proposal Metropolis with trained weights

Tolerances are the parity targets (max|dU| <= 1e-12 FP64 / 2e-6 FP32 after
the same PRN stream; plaquette 1e-13 / 1e-6 relative); the kernels and the
oracle perform the same operation sequence, so the links are also compared
bit for bit.  The oracle runs its per-link loops on all host cores; each
test prints the GPU and oracle wall times.
"""
import ctypes
import time

import numpy as np
import pytest

import _oracle as O
import qcdgpu_b200 as Q

pytestmark = pytest.mark.gpu

TOL_U = {0: 2e-6, 1: 1e-12}
TOL_P = {0: 1e-6, 1: 1e-13}
CHAIN_KEY1 = 0x5D3E1A27


def maxdiff(a, b):
    return float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64))))


def cfg_pair(group, dims, precision, beta, prng, start, n_or, reunit_every, reunit_fp64=1, instances=16384,
             seed=54):
    L = Q.Lattice(Q.default_config(group=group, size=dims, precision=precision, start=start, prng=prng, beta=beta,
                                   randseries=seed, prng_instances=instances, n_or=n_or, reunit_every=reunit_every,
                                   reunit_fp64=reunit_fp64))
    c = O.make_cfg(group=group, dims=dims, precision=precision, beta=beta, row_align=L.cfg.row_align)
    return L, c


def oracle_or_sweeps(c, t, n):
    for _ in range(n):
        for par in (1, 0):
            for mu in range(4):
                O.lib.ol_phase_or(ctypes.byref(c), O.vp(t), par, mu)


def check_plaquette(L, c, t, precision):
    sp, tp = L.plaquette_sums()
    osp, otp = O.plaquette(c, t)
    assert abs(sp - osp) <= TOL_P[precision] * abs(osp) and abs(tp - otp) <= TOL_P[precision] * abs(otp), \
        ((sp, tp), (osp, otp))


class Clock:
    def __init__(self):
        self.gpu = self.oracle = 0.0

    def g(self, fn, *a):
        t0 = time.time()
        r = fn(*a)
        self.gpu += time.time() - t0
        return r

    def o(self, fn, *a):
        t0 = time.time()
        r = fn(*a)
        self.oracle += time.time() - t0
        return r

    def report(self, what):
        print("%s: GPU %.2f s, oracle %.2f s" % (what, self.gpu, self.oracle))


# ------------------------------------------------ SU(2) 8^4 beta = 2.3, FP64
def test_su2_8x4_ranlux_hot_start_hb_2or():
    """The reference's RANLUX stream and hot start (lattice_random2 fed by the
    batch), 3 sweeps of 1 heatbath + 2 overrelaxation with the reference's
    Gram-Schmidt every sweep: links within 1e-12 of the oracle (bit-exact
    expected), plaquette within 1e-13"""
    clk = Clock()
    L, c = cfg_pair(2, (8, 8, 8, 8), 1, 2.3, Q.PRNG_RANLUX, Q.START_HOT, n_or=2, reunit_every=1, reunit_fp64=0)
    info = L.info()
    S = info.prng_samples
    R = O.Ranlux(54, L.cfg.prng_instances)
    clk.g(L.seed, 54)
    clk.g(L.init, Q.START_HOT)
    R.batch(S)                                   # PRNG::initialize's produce()
    t = O.new_table(c)
    for mu in range(4):
        clk.o(O.lib.ol_init_hot_dir, ctypes.byref(c), O.vp(t), mu, O.vp(R.batch(S)))
    assert np.array_equal(L.download(), t)
    for s in range(3):
        clk.g(L.sweep, 1)
        for par in (1, 0):
            for mu in range(4):
                clk.o(O.phase_hb, c, t, par, mu, R.batch(S))
        clk.o(oracle_or_sweeps, c, t, 2)
        clk.o(O.lib.ol_gramschmidt, ctypes.byref(c), O.vp(t))
        g = L.download()
        assert maxdiff(g, t) <= TOL_U[1], (s, maxdiff(g, t))
        assert np.array_equal(g, t), (s, maxdiff(g, t))
    check_plaquette(L, c, t, 1)
    clk.report("SU(2) 8^4 RANLUX 3 sweeps")


def test_su2_8x4_philox_haar_start_hb_2or():
    """The run configuration's own settings (Philox stream, Haar start, FP64
    reunitarisation every 10 sweeps): the oracle starts from the GPU's Haar
    field and follows 12 sweeps, one of them with the Gram-Schmidt pass"""
    clk = Clock()
    L, c = cfg_pair(2, (8, 8, 8, 8), 1, 2.3, Q.PRNG_PHILOX, Q.START_HAAR, n_or=2, reunit_every=10)
    clk.g(L.seed, 54)
    clk.g(L.init, Q.START_HAAR)
    t = L.download()
    ph = L.info().phase_counter
    for s in range(12):
        clk.g(L.sweep, 1)
        for par in (1, 0):
            for mu in range(4):
                clk.o(O.phase_hb, c, t, par, mu, None, (54, CHAIN_KEY1, ph))
                ph += 1
        clk.o(oracle_or_sweeps, c, t, 2)
        if (s + 1) % 10 == 0:
            clk.o(O.lib.ol_gramschmidt_fp64, ctypes.byref(c), O.vp(t))
    g = L.download()
    assert np.array_equal(g, t), maxdiff(g, t)
    check_plaquette(L, c, t, 1)
    assert L.info().phase_counter == ph
    clk.report("SU(2) 8^4 Philox 12 sweeps")


# ------------------------------------------ SU(3) 24^3 x 6 beta = 5.9, FP32
@pytest.mark.parametrize("prng", [Q.PRNG_PHILOX, Q.PRNG_RANLUX])
def test_su3_24x6_fp32_hb_4or(prng):
    """Two full sweeps of 1 heatbath + 4 overrelaxation from a cold start:
    FP32 links within 2e-6 of the oracle (bit-exact expected), plaquette
    within 1e-6 relative, for the Philox stream and the reference's RANLUX
    stream (one batch per heatbath phase)"""
    clk = Clock()
    dims = (24, 24, 24, 6)
    L, c = cfg_pair(3, dims, 0, 5.9, prng, Q.START_COLD, n_or=4, reunit_every=10)
    info = L.info()
    S = info.prng_samples
    R = O.Ranlux(54, L.cfg.prng_instances) if prng == Q.PRNG_RANLUX else None
    clk.g(L.seed, 54)
    clk.g(L.init, Q.START_COLD)
    if R is not None:
        R.batch(S)
    t = O.new_table(c)
    O.lib.ol_init_cold(ctypes.byref(c), O.vp(t))
    ph = 0
    for s in range(2):
        clk.g(L.sweep, 1)
        for par in (1, 0):
            for mu in range(4):
                if R is not None:
                    clk.o(O.phase_hb, c, t, par, mu, R.batch(S))
                else:
                    clk.o(O.phase_hb, c, t, par, mu, None, (54, CHAIN_KEY1, ph))
                ph += 1
        clk.o(oracle_or_sweeps, c, t, 4)
        g = L.download()
        assert maxdiff(g, t) <= TOL_U[0], (s, maxdiff(g, t))
        assert np.array_equal(g, t), (s, maxdiff(g, t))
    check_plaquette(L, c, t, 0)
    clk.report("SU(3) 24^3x6 %s 2 sweeps" % ("RANLUX" if R is not None else "Philox"))


# ------------------------------------------- SU(3) 32^4 beta = 6.0, FP32
def test_su3_32x4_bench_sweep_tuned_shapes():
    """The benchmark's lattice and settings: cold start, 2 sweeps, the launch
    shapes the tuner picks, then one timed-style sweep (8 heatbath + 32
    overrelaxation phases) against the oracle from the same field, then the
    FP64 Gram-Schmidt pass; links bit-exact (<= 2e-6 required), plaquette
    within 1e-6 relative"""
    clk = Clock()
    L, c = cfg_pair(3, (32, 32, 32, 32), 0, 6.0, Q.PRNG_PHILOX, Q.START_COLD, n_or=4, reunit_every=10)
    clk.g(L.seed, 54)
    clk.g(L.init, Q.START_COLD)
    clk.g(L.sweep, 2)
    clk.g(L.tune, 2)
    hb, orx = L.shapes()
    t = L.download()
    ph = L.info().phase_counter
    assert ph == 16
    clk.g(L.sweep, 1)
    for par in (1, 0):
        for mu in range(4):
            clk.o(O.phase_hb, c, t, par, mu, None, (54, CHAIN_KEY1, ph))
            ph += 1
    clk.o(oracle_or_sweeps, c, t, 4)
    g = L.download()
    d = maxdiff(g, t)
    assert d <= TOL_U[0], d
    assert np.array_equal(g, t), d
    check_plaquette(L, c, t, 0)
    clk.g(L.reunitarize, True)
    clk.o(O.lib.ol_gramschmidt_fp64, ctypes.byref(c), O.vp(t))
    assert np.array_equal(L.download(), t)
    clk.report("SU(3) 32^4 bench sweep, shapes HB %d OR %d" % (hb, orx))


@pytest.mark.parametrize("shape", range(Q.TUNE_SHAPES))
def test_su3_32x4_every_shape_one_phase_each(shape):
    """Every launch shape at 32^4 (the tuner may pick any of them): one
    heatbath and one overrelaxation phase on a thermalising field, bit for
    bit the oracle's"""
    clk = Clock()
    L, c = cfg_pair(3, (32, 32, 32, 32), 0, 6.0, Q.PRNG_PHILOX, Q.START_COLD, n_or=0, reunit_every=0)
    clk.g(L.seed, 54)
    clk.g(L.init, Q.START_COLD)
    clk.g(L.sweep, 1)
    L.set_shapes(shape, shape)
    t = L.download()
    ph = L.info().phase_counter
    clk.g(L.phase, 1, 2, Q.HEATBATH)
    clk.o(O.phase_hb, c, t, 1, 2, None, (54, CHAIN_KEY1, ph))
    clk.g(L.phase, 0, 3, Q.OVERRELAX)
    clk.o(O.lib.ol_phase_or, ctypes.byref(c), O.vp(t), 0, 3)
    g = L.download()
    assert np.array_equal(g, t), maxdiff(g, t)
    clk.report("SU(3) 32^4 shape %d, one HB + one OR phase" % shape)


# --------------------------- SU(3) 16^4 beta = 5.7, learned proposal, FP32
def test_su3_16x4_learned_metropolis_sweep_trained_weights():
    """The learned-proposal configuration: heatbath-thermalised 16^4 field,
    the network trained on the GPU for a few steps, then one Metropolis sweep
    (8 phases, 2 hits per subgroup): the tensor-core network's steps against
    the oracle's (BF16 operand roundings mirrored; bounds as in
    test_gpu_learned.py), and each phase bit for bit the oracle's given the
    GPU's steps, with the same trained weights and Philox stream"""
    clk = Clock()
    dims = (16, 16, 16, 16)
    L = Q.Lattice(Q.default_config(group=3, size=dims, precision=0, start=Q.START_COLD, prng=Q.PRNG_PHILOX,
                                   beta=5.7, randseries=54, n_or=0, reunit_every=10))
    c = O.make_cfg(group=3, dims=dims, precision=0, beta=5.7, row_align=L.cfg.row_align)
    clk.g(L.seed, 54)
    clk.g(L.init, Q.START_COLD)
    clk.g(L.sweep, 20)
    eps_max = 1.5
    L.net_set(Q.net_init(seed=2, out_bias=-0.4), eps_max)
    for _ in range(4):
        clk.g(L.sweep, 1)
        clk.g(L.net_train, 2, 2e-3)
    w, wb = L.net_get()
    assert np.array_equal(wb, Q.bf16_round(w))
    t = L.download()
    ph = L.info().phase_counter
    L.mh_stats(reset=True)
    acc = 0
    for k, (par, mu) in enumerate([(p, m) for p in (1, 0) for m in range(4)]):
        eps = clk.g(L.net_eps, par, mu)
        if k == 0:
            d = np.abs(eps.astype(np.float64) - O.net_eps(c, t, par, mu, wb, eps_max)) / eps_max
            print("eps vs oracle: max %.3g, 99.9%% %.3g" % (d.max(), np.quantile(d, 0.999)))
            assert np.quantile(d, 0.999) <= 1e-5 and d.max() <= 2e-2
        clk.g(L.mh_phase, par, mu, 2)
        a, _ = clk.o(O.mh_phase_eps, c, t, par, mu, eps, 2, 54, ph + k)
        acc += a
    g = L.download()
    assert np.array_equal(g, t), maxdiff(g, t)
    rate, _, hits = L.mh_stats()
    assert hits == O.volume(c) // 2 * 8 * 3 * 2 and round(rate * hits) == acc
    check_plaquette(L, c, t, 0)
    clk.report("SU(3) 16^4 learned Metropolis sweep (acceptance %.3f)" % rate)
