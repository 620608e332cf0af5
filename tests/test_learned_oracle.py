"""The learned proposal on the CPU (no GPU): the oracle's analytic gradient
of the training loss (ESJD) agrees with finite differences of the loss,
the BF16 rounding and constant-step helpers do what they say, and the
exp routine of the acceptance step is accurate."""
import math

import numpy as np
import pytest

import _oracle as O
import qcdgpu_b200 as Q


def thermal_table(dims=(4, 4, 4, 4), beta=5.7, sweeps=4, seed=77):
    c = O.make_cfg(group=3, dims=dims, precision=0, beta=beta, row_align=64)
    t = O.new_table(c)
    O.lib.ol_init_cold(O.ctypes.byref(c), O.vp(t))
    ph = 0
    for _ in range(sweeps):
        for par in (1, 0):
            for mu in range(4):
                O.phase_hb(c, t, par, mu, philox=(seed, O.CHAIN_KEY1, ph))
                ph += 1
        O.lib.ol_gramschmidt(O.ctypes.byref(c), O.vp(t))
    return c, t


def test_exp_routine_accuracy():
    for x in np.linspace(-30, 30, 601):
        assert abs(O.lib.ol_expd(float(x)) / math.exp(x) - 1) < 4e-16
    assert O.lib.ol_expd(0.0) == 1.0


def test_bf16_round_and_constant_step():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-3, 65504.0], dtype=np.float32)
    b = Q.bf16_round(a)
    assert b[0] == 1.0 and b[1] == 1.0                  # tie to even (mantissa ...0)
    assert b[2] == np.float32(1.0078125)                # above the tie rounds up
    assert np.all(np.abs(b - a) <= np.abs(a) * 2 ** -8)
    assert np.array_equal(Q.bf16_round(b), b)
    w = Q.net_constant(0.3, 1.2)
    x = np.random.default_rng(0).standard_normal(8).astype(np.float32)
    o = O.lib.ol_mlp_out(O._fp(np.ascontiguousarray(Q.bf16_round(w))), O._fp(x))
    assert abs(1.2 / (1 + math.exp(-o)) - 0.3) < 3e-3     # BF16 bias


def links_of(c, t):
    """reference-layout table -> complex U[gid, mu, 3, 3]"""
    V = O.volume(c)
    a = t.reshape(12, c.rowsize, 4)[:, :V, :].astype(np.float64)
    U = np.zeros((V, 4, 3, 3), dtype=np.complex128)
    for mu in range(4):
        p1, p2, p3 = a[mu], a[mu + 4], a[mu + 8]
        U[:, mu, 0, :] = p1[:, :3] + 1j * p2[:, :3]
        U[:, mu, 1, 0] = p3[:, 0] + 1j * p3[:, 2]
        U[:, mu, 1, 1] = p3[:, 1] + 1j * p3[:, 3]
        U[:, mu, 1, 2] = p1[:, 3] + 1j * p2[:, 3]
        U[:, mu, 2, :] = np.conj(np.cross(U[:, mu, 0, :], U[:, mu, 1, :]))
    return U


def table_of(c, U, dtype=np.float32):
    V = O.volume(c)
    a = np.zeros((12, c.rowsize, 4))
    for mu in range(4):
        a[mu, :V, :3], a[mu + 4, :V, :3] = U[:, mu, 0, :].real, U[:, mu, 0, :].imag
        a[mu, :V, 3], a[mu + 4, :V, 3] = U[:, mu, 1, 2].real, U[:, mu, 1, 2].imag
        a[mu + 8, :V] = np.stack([U[:, mu, 1, 0].real, U[:, mu, 1, 1].real, U[:, mu, 1, 0].imag,
                                  U[:, mu, 1, 1].imag], axis=1)
    return a.reshape(-1).astype(dtype)


def shift(c, gid, mu):
    n = list(c.n)
    x = [0, 0, 0, 0]
    y_, r = gid % n[1], gid // n[1]
    z_, r = r % n[2], r // n[2]
    t_, x_ = r % n[3], r // n[3]
    x = [x_, y_, z_, t_]
    x[mu] = (x[mu] + 1) % n[mu]
    return x[1] + n[1] * (x[2] + n[2] * (x[3] + n[3] * x[0]))


def random_su3(rng, k):
    z = rng.standard_normal((k, 3, 3)) + 1j * rng.standard_normal((k, 3, 3))
    q, r = np.linalg.qr(z)
    q = q * (np.diagonal(r, axis1=1, axis2=2) / np.abs(np.diagonal(r, axis1=1, axis2=2)))[:, None, :]
    return q / np.linalg.det(q)[:, None, None] ** (1 / 3)


def test_features_are_gauge_invariant_and_bounded():
    c, t = thermal_table()
    V = O.volume(c)
    rng = np.random.default_rng(4)
    U = links_of(c, t)
    g = random_su3(rng, V)
    Ug = np.empty_like(U)
    for s in range(V):
        for mu in range(4):
            Ug[s, mu] = g[s] @ U[s, mu] @ g[shift(c, s, mu)].conj().T
    tg = table_of(c, Ug)
    for gid in rng.integers(0, V, 6):
        for mu in range(4):
            x = O.mh_features(c, t, int(gid), mu)
            assert 0 < x[0] <= 1 and 1 / 3 - 1e-6 <= x[1] <= 1 + 1e-6
            assert abs(x[2]) <= 1 + 1e-5 and abs(x[3]) <= 1 + 1e-5
            assert abs(x[4]) <= 1 + 1e-5 and 0 <= x[5] <= 1 + 1e-5
            xg = O.mh_features(c, tg, int(gid), mu)
            assert np.max(np.abs(x - xg)) < 2e-5, (x, xg)


def test_analytic_gradient_matches_finite_differences():
    c, t = thermal_table()
    w = Q.bf16_round(Q.net_init(seed=3, out_bias=-0.5)).astype(np.float64)
    eps_max, key, phase = 1.0, 9, 5
    g, st = O.mh_grad(c, t, 1, 2, w.astype(np.float32), eps_max, key, phase)
    assert st[3] == O.volume(c) // 2 and 0 < st[2] <= 1 and st[1] > 0 and abs(st[0] + st[1]) < 1e-12
    loss0 = O.mh_loss(c, t, 1, 2, w, eps_max, key, phase)
    assert abs(loss0 - st[0]) < 1e-5 * abs(st[0])
    rng = np.random.default_rng(1)
    idx = list(rng.choice(Q.NET_PARAMS - 1, 14, replace=False)) + [Q.NET_PARAMS - 1]
    h = 1e-4
    for q in idx:
        wp, wm = w.copy(), w.copy()
        wp[q] += h
        wm[q] -= h
        fd = (O.mh_loss(c, t, 1, 2, wp, eps_max, key, phase) - O.mh_loss(c, t, 1, 2, wm, eps_max, key, phase)) / (2 * h)
        assert abs(fd - g[q]) <= 2e-3 * max(abs(fd), 1e-3), (q, fd, g[q])


def test_tensor_core_definition_close_to_fp32_network():
    """The oracle's restatement of the tensor-core network (BF16 features and
    hidden layer, FP32 sums) stays within BF16 rounding of the FP32 network:
    per-link steps to 1 % of eps_max, the gradient to a few per cent in norm"""
    c, t = thermal_table()
    w = Q.bf16_round(Q.net_init(seed=4, out_bias=0.1))
    e_tc = O.net_eps(c, t, 1, 3, w, 1.5)
    assert e_tc.shape == (O.volume(c) // 2,) and np.all(e_tc > 0) and np.all(e_tc < 1.5)
    x = np.array([O.mh_features(c, t, g, 3) for g in range(O.volume(c))])
    assert np.all(np.isfinite(x))
    g_tc, _ = O.mh_grad(c, t, 1, 3, w, 1.5, 9, 2, tc=True)
    g_32, _ = O.mh_grad(c, t, 1, 3, w, 1.5, 9, 2, tc=False)
    assert np.linalg.norm(g_tc - g_32) <= 0.05 * np.linalg.norm(g_32)
    # the constant-step network has no hidden contribution: both definitions agree exactly
    wc = Q.net_constant(0.4, 1.5)
    assert np.allclose(O.net_eps(c, t, 0, 1, wc, 1.5), 0.4, rtol=1e-2)
