"""The learned-proposal Metropolis update on the GPU against the oracle.

The network runs on the tcgen05 tensor cores (BF16 operands, FP32
accumulation in tensor memory); the oracle restates it with the same BF16
roundings and sums in order, so the step eps agrees to FP32 accumulation
error -- except for the rare link where that error moves a hidden value
across a BF16 rounding boundary (one BF16 unit, 2^-8 relative, in one
hidden unit).  Bounds: |d eps| <= 1e-5 eps_max for 99.9 % of the links and
<= 2e-2 eps_max for all.  Given the GPU's eps, one Metropolis phase
reproduces the oracle's chain bit for bit (same Philox stream); a sweep
equals its phases; the training gradient agrees with the oracle's (same
roundings) to 1e-3 in norm; a learned chain samples the heatbath's
plaquette (exactness, within 2 sigma with tau_int); training raises the
jump distance above the best constant step."""
import json
import os

import numpy as np
import pytest

import _oracle as O
import qcdgpu_b200 as Q

pytestmark = pytest.mark.gpu

DIMS = (4, 4, 4, 8)
SERIES = 21


def thermal(beta=5.7, sweeps=3, dims=DIMS):
    L = Q.Lattice(Q.default_config(group=3, size=dims, precision=0, start=Q.START_HOT, prng=Q.PRNG_PHILOX,
                                   beta=beta, randseries=SERIES, row_align=64, n_or=0, reunit_every=0))
    L.seed(SERIES)
    L.init()
    L.sweep(sweeps)
    c = O.make_cfg(group=3, dims=dims, precision=0, beta=beta, row_align=64)
    return L, c


def check_eps(got, ref, eps_max):
    d = np.abs(got.astype(np.float64) - ref.astype(np.float64)) / eps_max
    q = float(np.quantile(d, 0.999))
    print("eps vs oracle: max %.3g, 99.9%% %.3g (units of eps_max), %d links" % (d.max(), q, d.size))
    assert q <= 1e-5 and d.max() <= 2e-2
    return d


@pytest.mark.parametrize("parity,mu,nhit,eps_max", [(1, 2, 2, 1.0), (0, 0, 1, 2.5), (1, 3, 3, 0.4)])
def test_mh_phase_matches_oracle(parity, mu, nhit, eps_max):
    L, c = thermal()
    w = Q.bf16_round(Q.net_init(seed=mu + 10, out_bias=0.3))
    L.net_set(w, eps_max)
    m, b = L.net_get()
    assert np.array_equal(b, w) and np.array_equal(m, w)
    tab = L.download()
    ph = L.info().phase_counter
    eps = L.net_eps(parity, mu)
    assert np.array_equal(L.download(), tab)              # eps alone changes nothing
    check_eps(eps, O.net_eps(c, tab, parity, mu, w, eps_max), eps_max)
    L.mh_stats(reset=True)
    L.mh_phase(parity, mu, nhit)
    acc, jump = O.mh_phase_eps(c, tab, parity, mu, eps, nhit, SERIES, ph)
    got = L.download()
    assert np.array_equal(got, tab)
    rate, j, hits = L.mh_stats()
    assert hits == O.volume(c) // 2 * 3 * nhit
    assert round(rate * hits) == acc and 0 < acc < hits
    assert abs(j * hits - jump) <= 1e-9 * jump
    assert L.info().phase_counter == ph + 1


def test_mh_sweep_equals_its_phases_and_the_oracle():
    """two learned-proposal sweeps on one context equal, bit for bit, the
    same 16 phases run one by one on a second context; each of those phases
    equals the oracle's given the GPU's eps"""
    L, c = thermal()
    L2, _ = thermal()
    w = Q.bf16_round(Q.net_init(seed=5, out_bias=-0.2))
    L.net_set(w, 1.2)
    L2.net_set(w, 1.2)
    tab = L2.download()
    ph = L2.info().phase_counter
    L.mh_sweep(2, 1)
    k = 0
    for s in range(2):
        for par in (1, 0):
            for mu in range(4):
                eps = L2.net_eps(par, mu)
                L2.mh_phase(par, mu, 1)
                O.mh_phase_eps(c, tab, par, mu, eps, 1, SERIES, ph + k)
                k += 1
                assert np.array_equal(L2.download(), tab), (s, par, mu)
    assert np.array_equal(L.download(), L2.download())


def test_training_gradient_matches_oracle():
    L, c = thermal()
    w = Q.bf16_round(Q.net_init(seed=3, out_bias=-0.5))
    L.net_set(w, 1.0)
    tab = L.download()
    for k, (par, mu) in enumerate([(1, 2), (0, 1)]):
        g, st = L.net_grad(par, mu)
        go, sto = O.mh_grad(c, tab, par, mu, w, 1.0, SERIES, k, tc=True)
        gx, _ = O.mh_grad(c, tab, par, mu, w, 1.0, SERIES, k, tc=False)
        r = np.linalg.norm(g - go) / np.linalg.norm(go)
        print("gradient vs oracle (same roundings) %.3g; BF16 operands vs FP32 network %.3g"
              % (r, np.linalg.norm(go - gx) / np.linalg.norm(gx)))
        assert r <= 1e-3
        assert abs(st[0] - sto[0]) <= 1e-5 * abs(sto[0]) and abs(st[2] - sto[2]) <= 1e-5
        assert st[3] == sto[3] == O.volume(c) // 2
    assert np.array_equal(L.download(), tab)               # training reads the field only


def test_adam_step_moves_master_and_keeps_bf16_copy():
    L, c = thermal()
    w = Q.bf16_round(Q.net_init(seed=2))
    L.net_set(w, 1.0)
    st = L.net_train(3, 1e-2)
    m, b = L.net_get()
    assert not np.array_equal(m, w)
    assert np.array_equal(b, Q.bf16_round(m))
    assert st[3] == O.volume(c) // 2 and st[1] > 0


def test_learned_chain_samples_the_heatbath_plaquette():
    """exactness: a chain of learned-proposal sweeps (random, untrained
    weights -- any weights keep the chain exact) agrees with the reference
    heatbath's long-run plaquette at SU(3) 4^4 beta=5.7"""
    gold = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "stat_parity.json")))
    case = [c for c in gold["cases"] if c["name"] == "su3_4x4_b5.7"][0]
    L = Q.Lattice(Q.default_config(group=3, size=(4, 4, 4, 4), precision=0, start=Q.START_COLD,
                                   prng=Q.PRNG_PHILOX, beta=5.7, randseries=31, n_or=0, reunit_every=10))
    L.seed(31)
    L.init()
    L.net_set(Q.net_init(seed=1, out_bias=0.0), 1.2)
    L.mh_sweep(500, 2)
    n = 12000
    p = np.zeros(n)
    for i in range(n):
        L.mh_sweep(1, 2)
        sp, tp = L.plaquette_sums()
        p[i] = (sp + tp) / (6 * 256)
    tau, _ = Q.tau_int(p)
    err = np.sqrt(2 * tau * p.var() / n)
    z = (p.mean() - case["mean"]) / np.hypot(err, case["error"])
    acc = L.mh_stats()[0]
    print("learned chain: %.6f +- %.6f (tau %.2f, acceptance %.3f), reference %.6f +- %.6f, z = %.2f"
          % (p.mean(), err, tau, acc, case["mean"], case["error"], z))
    assert 0.1 < acc < 0.95 and abs(z) <= 2.0


def test_training_beats_the_best_constant_step():
    L = Q.Lattice(Q.default_config(group=3, size=(8, 8, 8, 8), precision=0, start=Q.START_COLD,
                                   prng=Q.PRNG_PHILOX, beta=5.7, randseries=41, n_or=0, reunit_every=10))
    L.seed(41)
    L.init()
    L.sweep(60)
    eps_max = 1.5

    def esjd(w, reps=2):
        L.net_set(w, eps_max)
        return np.mean([L.net_grad(p, m)[1][1] for _ in range(reps) for p in (1, 0) for m in range(4)])

    grid = [0.2, 0.3, 0.4, 0.5, 0.6, 0.75, 0.9]
    scan = [esjd(Q.net_constant(e, eps_max)) for e in grid]
    best = grid[int(np.argmax(scan))]
    r = best / eps_max
    L.net_set(Q.net_init(seed=2, out_bias=float(np.log(r / (1 - r)))), eps_max)
    for _ in range(150):
        L.sweep(1)
        L.net_train(2, 2e-3)
    trained, _ = L.net_get()
    e_t, e_c = [], []
    for _ in range(6):
        L.sweep(2)
        e_t.append(esjd(trained, 1))
        e_c.append(esjd(Q.net_constant(best, eps_max), 1))
    gain = np.mean(e_t) / np.mean(e_c) - 1
    print("best constant step %.2f: ESJD %.4f; trained ESJD %.4f; gain %.3f" % (best, np.mean(e_c), np.mean(e_t),
                                                                                gain))
    assert gain > 0.0
