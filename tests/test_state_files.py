"""Lattice state files (.qcg) and the tau_int estimator, host side (no GPU).

The file layout is checked word by word against the reference's writer
(SU(N)/suncl/suncl.cpp:1857-2079, lattice_make_bin_header): the test parses
the bytes itself with numpy, independently of the library's reader."""
import numpy as np
import pytest

import qcdgpu_b200 as Q


def word(s):
    b = s.encode()[:4].ljust(4, b"\0")
    return int.from_bytes(b, "little")


def make_table(cfg, rng):
    V = int(np.prod(list(cfg.size)))
    a = cfg.row_align
    rowsize = (V + a - 1) // a * a
    n = (12 if cfg.group == 3 else 4) * rowsize * 4
    return rng.standard_normal(n).astype(np.float64 if cfg.precision else np.float32)


@pytest.mark.parametrize("group,precision,prng", [(3, 0, Q.PRNG_RANLUX), (3, 1, Q.PRNG_PHILOX),
                                                  (2, 1, Q.PRNG_RANLUX)])
def test_state_file_layout_and_roundtrip(tmp_path, group, precision, prng):
    rng = np.random.default_rng(5)
    cfg = Q.default_config(group=group, size=(4, 6, 4, 8), precision=precision, prng=prng, beta=5.9, phi=0.25,
                           omega=-0.5, nhit=7, randseries=1234, ranlux_nskip=97, row_align=64, n_or=3,
                           reunit_every=10, reunit_fp64=1, wilson_r=3, wilson_t=2, start=Q.START_HOT)
    st = Q.RunState(init=1, nav=20, nav_counter=20, niter=5, iter=9, iter_counter=6, pl_level=3, get_actions=1,
                    get_plaquettes=1, get_wilson=1, prng_counter=331, phase_counter=(1 << 40) + 17,
                    sweeps_done=45, fmunu=1, fmunu_index1=3, fmunu_index2=8 if group == 3 else 2,
                    get_actions_diff=1)
    n = st.iter
    prow = Q.profile_row(cfg, st)
    assert prow == 2 * 2 * (4 + 6 + 4)
    series = {"actions": rng.standard_normal(2 * n), "plaquettes": rng.standard_normal(2 * n),
              "wilson": rng.standard_normal(n), "polyakov": rng.standard_normal(4 * n),
              "fmunu_series": rng.standard_normal(12 * n), "profiles": rng.standard_normal(prow * n)}
    table = make_table(cfg, rng)
    path = str(tmp_path / "s.qcg")
    Q.write_state_file(path, cfg, st, table, series)

    raw = open(path, "rb").read()
    h = np.frombuffer(raw[:256], dtype="<u4")
    assert h[0] == word("QCDG") and h[1] == word("PU") and h[2] == word("1.5") and h[3] == 0
    assert h[4] == 1 and h[5] == Q.START_HOT and h[6] == 1234
    assert h[7] == (12 if prng == Q.PRNG_PHILOX else 4) and h[8] == 97 and h[9] == 331
    assert list(h[10:18]) == [20, 20, 5, 9, 6, 7, 3, 2]
    assert h[18] == (2 if precision else 1)
    assert np.frombuffer(h[19:21].tobytes(), "<f8")[0] == 5.9
    assert np.frombuffer(h[21:23].tobytes(), "<f8")[0] == 0.25
    assert np.frombuffer(h[23:25].tobytes(), "<f8")[0] == -0.5
    assert list(h[25:32]) == [3, 3, 8 if group == 3 else 2, 1, 1, 1, 1]
    meas_F, en, en_F, pol = (int(x) for x in h[32:36])
    assert en == 64 and en_F == 7 * 64 and pol == 64          # MODEL_energies_size = 7
    assert h[36] == group and h[37] == 4 and list(h[38:42]) == [4, 6, 4, 8] and list(h[42:46]) == [4, 6, 4, 8]
    assert h[48] == word("B200") and h[60] == 1 and h[61] == 1

    # buffers in the reference's order: measurement, energies, energies_plq,
    # wilson loop, polyakov loop, link table
    off = 256 + 16 * meas_F
    e = np.frombuffer(raw[off:off + 16 * en], "<f8").reshape(-1, 2)
    off += 16 * en
    p = np.frombuffer(raw[off:off + 16 * en_F], "<f8").reshape(-1, 2)
    off += 16 * en_F
    w = np.frombuffer(raw[off:off + 8 * en], "<f8")
    off += 8 * en
    pl = np.frombuffer(raw[off:off + 16 * pol], "<f8").reshape(-1, 2)
    off += 16 * pol
    k = st.iter_counter
    assert np.array_equal(e[:k].ravel(), series["actions"][:2 * k]) and not e[k:].any()
    assert np.array_equal(p[:k].ravel(), series["plaquettes"][:2 * k])
    # F_munu in energies_plq blocks 1..6: index1 planes xy, xz, yz, then index2
    f = series["fmunu_series"].reshape(-1, 6, 2)
    for b in range(6):
        assert np.array_equal(p[(b + 1) * en:(b + 1) * en + k], f[:k, b]), b
    assert np.array_equal(w[:k], series["wilson"][:k])
    assert np.array_equal(pl[:k], series["polyakov"].reshape(-1, 4)[:k, :2])
    t = np.frombuffer(raw[off:off + table.nbytes], table.dtype)
    assert np.array_equal(t, table)
    off += table.nbytes
    assert np.frombuffer(raw[off:off + 4], "<u4")[0] == word("QGP4")
    off += 4 + 16 * pol
    assert np.frombuffer(raw[off:off + 4], "<u4")[0] == word("QGPF")
    prof = np.frombuffer(raw[off + 4:off + 4 + 8 * prow * en], "<f8").reshape(en, prow)
    assert np.array_equal(prof[:k], series["profiles"].reshape(n, prow)[:k]) and not prof[k:].any()
    assert len(raw) == off + 4 + 8 * prow * en

    cfg2, st2, ser2, table2 = Q.read_state_file(path)
    assert np.array_equal(table2, table)
    for f in ("group", "precision", "start", "randseries", "prng", "ranlux_nskip", "nhit", "wilson_r", "wilson_t",
              "n_or", "reunit_every", "reunit_fp64", "row_align"):
        assert getattr(cfg2, f) == getattr(cfg, f), f
    assert list(cfg2.size) == list(cfg.size)
    assert (cfg2.beta, cfg2.phi, cfg2.omega) == (cfg.beta, cfg.phi, cfg.omega)
    for f in ("init", "nav", "nav_counter", "niter", "iter", "iter_counter", "pl_level", "prng_counter",
              "phase_counter", "sweeps_done"):
        assert getattr(st2, f) == getattr(st, f), f
    for f in ("fmunu", "fmunu_index1", "fmunu_index2", "get_actions_diff"):
        assert getattr(st2, f) == getattr(st, f), f
    for key, m in (("actions", 2), ("plaquettes", 2), ("wilson", 1), ("polyakov", 4), ("fmunu_series", 12),
                   ("profiles", prow)):
        assert np.array_equal(ser2[key][:m * k], series[key][:m * k]), key


def test_state_file_rejects_foreign_and_truncated(tmp_path):
    bad = tmp_path / "bad.qcg"
    bad.write_bytes(b"NOTQCDGPU" + b"\0" * 400)
    with pytest.raises(Q.QGError):
        Q.read_state_file(str(bad))
    rng = np.random.default_rng(1)
    cfg = Q.default_config(group=3, size=(4, 4, 4, 4), precision=0, row_align=64)
    st = Q.RunState(init=1, nav=0, niter=1, iter=2, iter_counter=2, pl_level=1, get_actions=1, get_plaquettes=1)
    good = str(tmp_path / "good.qcg")
    Q.write_state_file(good, cfg, st, make_table(cfg, rng))
    raw = open(good, "rb").read()
    (tmp_path / "short.qcg").write_bytes(raw[:-100])
    with pytest.raises(Q.QGError):
        Q.read_state_file(str(tmp_path / "short.qcg"))
    with pytest.raises(Q.QGError):
        Q.write_state_file(str(tmp_path / "x.qcg"), cfg, st, np.zeros(10, np.float32))


def tau_numpy(x, c=6.0):
    """The Madras-Sokal automatic window, restated for the check."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    d = x - x.mean()
    c0 = np.dot(d, d) / n
    t = 0.5
    for w in range(1, n):
        t += np.dot(d[:-w], d[w:]) / n / c0
        if w >= c * t:
            return t, w
    return t, n - 1


def test_tau_int_matches_restatement_and_ar1_theory():
    rng = np.random.default_rng(3)
    for phi in (0.0, 0.5, 0.9):
        n = 100000
        e = rng.standard_normal(n)
        x = np.empty(n)
        x[0] = e[0]
        for i in range(1, n):
            x[i] = phi * x[i - 1] + e[i]
        t, w = Q.tau_int(x)
        t2, w2 = tau_numpy(x)
        assert w == w2 and abs(t - t2) < 1e-9
        exact = (1 + phi) / (2 * (1 - phi))
        assert abs(t - exact) < 0.08 * exact, (phi, t, exact)
    assert Q.tau_int([1.0]) == (0.5, 0)
    assert Q.tau_int([2.0] * 10) == (0.5, 0)


def test_init_file_state_keys(tmp_path):
    p = tmp_path / "init.dat"
    p.write_text("INIT = 0\nSTATEFILE = /x/y.qcg\nSAVESTATE = 1\nSAVEEVERY = 5\nSTATEOUT = out.qcg\n")
    cfg, opts = Q.parse_init_file(str(p))
    assert opts.init == 0 and opts.state_file == b"/x/y.qcg" and opts.save_state == 1
    assert opts.save_every_iter == 5 and opts.state_out == b"out.qcg"
    assert Q.default_run_options().init == 1
