"""The oracle's F_munu projections and action / Polyakov profiles against an
independent numpy restatement (plaquette matrices from the decoded link
table, -i Tr(P T_a) with the Gell-Mann / Pauli matrices written out), and
their consistency with the oracle's whole-lattice sums (CPU only).

Reference: the FMUNU / F0MU plaquette kernels (sun_measurements_cl.cl:
712-1175), trace_lambda1..8_double (su3_measurements_cl.cl:355-460),
trace_sigma1..3_double (su2_measurements_cl.cl:89-124), lattice_action_diff_*
(sun_measurements_cl.cl:187-615), lattice_polyakov_diff_* (polyakov.cl:
142-402).
"""
import numpy as np
import pytest

import _oracle as O

S3 = 1.0 / np.sqrt(3.0)
GELL_MANN = {
    1: [[0, 1, 0], [1, 0, 0], [0, 0, 0]],
    2: [[0, -1j, 0], [1j, 0, 0], [0, 0, 0]],
    3: [[1, 0, 0], [0, -1, 0], [0, 0, 0]],
    4: [[0, 0, 1], [0, 0, 0], [1, 0, 0]],
    5: [[0, 0, -1j], [0, 0, 0], [1j, 0, 0]],
    6: [[0, 0, 0], [0, 0, 1], [0, 1, 0]],
    7: [[0, 0, 0], [0, 0, -1j], [0, 1j, 0]],
    8: [[S3, 0, 0], [0, S3, 0], [0, 0, -2 * S3]],
}
PAULI = {1: [[0, 1], [1, 0]], 2: [[0, -1j], [1j, 0]], 3: [[1, 0], [0, -1]]}


def decode(c, tab):
    """links[x, y, z, t, mu] as complex N x N matrices"""
    n = list(c.n)
    V = int(np.prod(n))
    N = c.group
    U = np.zeros((n[0], n[1], n[2], n[3], 4, N, N), dtype=complex)
    if N == 3:
        a = tab.reshape(12, c.rowsize, 4)[:, :V, :].astype(np.float64)
    else:
        a = tab.reshape(4, c.rowsize, 4)[:, :V, :].astype(np.float64)
    for g in range(V):
        # gid = y + N2 z + N2 N3 t + N2 N3 N4 x
        y = g % n[1]
        z = (g // n[1]) % n[2]
        t = (g // (n[1] * n[2])) % n[3]
        x = g // (n[1] * n[2] * n[3])
        for mu in range(4):
            if N == 3:
                u1, u2, u3 = a[mu, g], a[mu + 4, g], a[mu + 8, g]
                r0 = np.array([u1[0] + 1j * u2[0], u1[1] + 1j * u2[1], u1[2] + 1j * u2[2]])
                r1 = np.array([u3[0] + 1j * u3[2], u3[1] + 1j * u3[3], u1[3] + 1j * u2[3]])
                U[x, y, z, t, mu] = np.array([r0, r1, np.conj(np.cross(r0, r1))])
            else:
                q = a[mu, g]
                p1, p2 = q[0] + 1j * q[2], q[1] + 1j * q[3]
                U[x, y, z, t, mu] = np.array([[p1, p2], [-np.conj(p2), np.conj(p1)]])
    return U


def shift(U, d):
    """U(x + d) as an array over x"""
    return np.roll(U, -1, axis=d)


def plaq(U, m, n):
    Um, Un = U[..., m, :, :], U[..., n, :, :]
    dag = lambda A: np.conj(np.swapaxes(A, -1, -2))
    return Um @ shift(Un, m) @ dag(shift(Um, n)) @ dag(Un)


def gid_table(c):
    t = O.new_table(c)
    O.lib.ol_init_gid(O.ctypes.byref(c), O.vp(t))
    return t


CASES = [(3, 1), (3, 0), (2, 1)]


@pytest.mark.parametrize("group,precision", CASES)
def test_fmunu_matches_generator_definition(group, precision):
    c = O.make_cfg(group=group, dims=(4, 4, 2, 6), precision=precision)
    t = gid_table(c)
    U = decode(c, t)
    gens = GELL_MANN if group == 3 else PAULI
    pairs = [(1, 5), (2, 6), (3, 8), (4, 7)] if group == 3 else [(1, 2), (3, 2)]
    for field, planes in ((0, [(0, 1), (0, 2), (1, 2)]), (1, [(0, 3), (1, 3), (2, 3)])):
        for i1, i2 in pairs:
            got = O.fmunu(c, t, field, i1, i2)
            for gi, a in enumerate((i1, i2)):
                T = np.array(gens[a], dtype=complex) / 2
                for p, (m, n) in enumerate(planes):
                    f = (-1j * np.trace(plaq(U, m, n) @ T, axis1=-2, axis2=-1)).sum()
                    if group == 2:
                        f = f.real            # the SU(2) projections are real by construction
                    assert abs(got[gi, p, 0] - f.real) < 1e-9, (field, a, p)
                    assert abs(got[gi, p, 1] - f.imag) < 1e-9, (field, a, p)


@pytest.mark.parametrize("group,precision", CASES)
def test_fmunu_vanishes_on_cold_start(group, precision):
    c = O.make_cfg(group=group, dims=(4, 4, 4, 4), precision=precision)
    t = O.new_table(c)
    O.lib.ol_init_cold(O.ctypes.byref(c), O.vp(t))
    for field in (0, 1):
        assert np.all(O.fmunu(c, t, field, 3, 8 if group == 3 else 2) == 0.0)


@pytest.mark.parametrize("group,precision", CASES)
def test_profiles_match_restatement_and_totals(group, precision):
    c = O.make_cfg(group=group, dims=(6, 4, 2, 4), precision=precision, beta=5.7)
    t = gid_table(c)
    U = decode(c, t)
    N = group
    bet = float(np.float32(c.beta / N)) if precision == 0 else c.beta / N
    rs = sum(np.trace(plaq(U, m, n), axis1=-2, axis2=-1).real for m, n in ((0, 1), (0, 2), (1, 2)))
    rt = sum(np.trace(plaq(U, m, n), axis1=-2, axis2=-1).real for m, n in ((0, 3), (1, 3), (2, 3)))
    s_site, t_site = bet * (3 * N - rs), bet * (3 * N - rt)
    act = O.action(c, t)
    pol = O.polyakov(c, t)
    # Polyakov loop per spatial site: ordered product along t
    P = U[:, :, :, 0, 3]
    for k in range(1, c.n[3]):
        P = P @ U[:, :, :, k, 3]
    trP = np.trace(P, axis1=-2, axis2=-1)
    for axis in range(3):
        ap = O.action_profile(c, t, axis)
        other = tuple(d for d in range(4) if d != axis)
        assert np.allclose(ap[:, 0], s_site.sum(axis=other), rtol=1e-9, atol=1e-9)
        assert np.allclose(ap[:, 1], t_site.sum(axis=other), rtol=1e-9, atol=1e-9)
        assert abs(ap[:, 0].sum() - act[0]) <= 1e-10 * abs(act[0]) + 1e-10
        assert abs(ap[:, 1].sum() - act[1]) <= 1e-10 * abs(act[1]) + 1e-10
        pp = O.polyakov_profile(c, t, axis)
        others = tuple(d for d in range(3) if d != axis)
        tol = 1e-5 if precision == 0 else 1e-10
        assert np.allclose(pp[:, 0], trP.real.sum(axis=others), rtol=tol, atol=tol)
        assert np.allclose(pp[:, 1], trP.imag.sum(axis=others), rtol=tol, atol=tol)
        assert abs(pp[:, 0].sum() - pol[0]) <= 1e-10 * (1 + abs(pol[0]))
        assert abs(pp[:, 1].sum() - pol[1]) <= 1e-10 * (1 + abs(pol[1]))
