"""The host driver end to end on the GPU (qg_run through the C-ABI): the
measurement series equals the oracle's for the same cadence, the CPU re-check
passes and the results file has the reference's layout."""
import ctypes
import os

import numpy as np
import pytest

import _oracle as O
import qcdgpu_b200 as Q

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("group,precision", [(3, 1), (3, 0), (2, 1)])
def test_run_gid_series_matches_oracle(tmp_path, group, precision):
    dims = (4, 4, 4, 4)
    cfg = Q.default_config(group=group, size=dims, precision=precision, start=Q.START_GID, beta=6.0,
                           prng_instances=512, row_align=64, wilson_r=2, wilson_t=2)
    opts = Q.default_run_options(iter=4, niter=2, nav=1, pl_level=2, get_wilson=1, quiet=1,
                                 output_path=str(tmp_path) + "/", prefix="su%d-" % group)
    res = Q.run(cfg, opts)
    assert res.verification_passed == 1
    c = O.make_cfg(group=group, dims=dims, precision=precision, beta=6.0, row_align=64, gid_mode=True)
    t = O.new_table(c)
    O.lib.ol_init_gid(ctypes.byref(c), O.vp(t))
    V = O.volume(c)

    def sweep():
        for par in (1, 0):
            for mu in range(4):
                O.phase_hb(c, t, par, mu, philox=(0, 0, 0))
        O.lib.ol_gramschmidt(ctypes.byref(c), O.vp(t))

    plq = []
    sp, tp = O.plaquette(c, t)
    plq.append((sp + tp) / (6 * V))
    sweep()                                              # NAV
    for i in range(1, 4):
        sweep(); sweep()                                 # NITER
        sp, tp = O.plaquette(c, t)
        plq.append((sp + tp) / (6 * V))
    tol = 1e-12 if precision else 1e-6
    assert abs(res.mean[Q.OBS_NAMES.index("Plq_total")] - np.mean(plq[1:])) <= tol
    assert abs(res.gpu_last[1] - plq[-1]) <= tol
    rows = [l for l in open(res.results_file.decode()).read().split("\n") if l[:5].strip().isdigit()]
    assert len(rows) == 4
    assert abs(float(rows[-1].split()[3]) - plq[-1]) <= max(tol, 1e-12)


def test_cli_runs_init_file(tmp_path):
    p = os.path.join(str(tmp_path), "init.dat")
    with open(p, "w") as f:
        f.write("GROUP = 3\nLS = 4\nLT = 4\nITER = 3\nNITER = 1\nNAV = 2\nBETA = 5.7\nINTS = 0\nRANDSERIES = 7\n"
                "PRNG = RANLUX3\nPRNG_INSTANCES = 256\nPRECISION = 1\nOUTPUTPATH = %s/\nPL_LEVEL = 2\n" % tmp_path)
    import subprocess
    exe = os.path.join(Q.PKG_DIR, "bin", "qcdgpu")
    out = subprocess.run([exe, p], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert "Verification successfully passed!" in out.stdout
    files = sorted(f for f in os.listdir(str(tmp_path)) if f.startswith("su3-") and f.endswith(".txt"))
    # the results file and its companion with this library's statistics
    main = [f for f in files if not f.endswith("-stats.txt")]
    assert len(files) == 2 and len(main) == 1 and main[0][:-4] + "-stats.txt" in files, files


@pytest.mark.parametrize("prng,start,precision", [(Q.PRNG_PHILOX, Q.START_HOT, 0), (Q.PRNG_RANLUX, Q.START_HOT, 0),
                                                  (Q.PRNG_RANLUX, Q.START_COLD, 1)])
def test_resume_from_state_file_continues_the_same_chain(tmp_path, prng, start, precision):
    """INIT = 0: a run stopped after ITER_counter = 3 and continued from its
    .qcg (RANLUX replayed to PRNG_counter, or the Philox counter restored)
    ends in the same link table and measured series as an uninterrupted
    run -- bit for bit."""
    import struct
    base = dict(group=3, size=(4, 4, 4, 8), precision=precision, start=start, prng=prng, beta=5.9,
                prng_instances=256, row_align=64, n_or=2, reunit_every=3, wilson_r=2, wilson_t=2)
    common = dict(niter=2, nav=3, pl_level=3, get_wilson=1, quiet=1, write_results=0, verify=0, save_state=1,
                  fmunu=1, get_actions_diff=1)
    full, half, resumed = (str(tmp_path / n) for n in ("full.qcg", "half.qcg", "resumed.qcg"))
    Q.run(Q.default_config(**base), Q.default_run_options(iter=6, state_out=full, **common))
    Q.run(Q.default_config(**base), Q.default_run_options(iter=3, state_out=half, **common))
    raw = bytearray(open(half, "rb").read())
    assert struct.unpack_from("<I", raw, 14 * 4)[0] == 3          # ITER_counter
    struct.pack_into("<I", raw, 13 * 4, 6)                         # extend ITER to 6
    open(half, "wb").write(bytes(raw))
    res = Q.run(Q.default_config(), Q.default_run_options(init=0, state_file=half, state_out=resumed, quiet=1,
                                                          write_results=0, verify=0, save_state=1))
    assert res.samples == 6
    c1, s1, ser1, t1 = Q.read_state_file(full)
    c2, s2, ser2, t2 = Q.read_state_file(resumed)
    assert s1.iter_counter == s2.iter_counter == 6
    assert s1.prng_counter == s2.prng_counter and s1.phase_counter == s2.phase_counter
    assert s1.sweeps_done == s2.sweeps_done == 3 + 5 * 2
    assert np.array_equal(t1, t2)
    for k in ser1:
        assert np.array_equal(ser1[k], ser2[k]), k


@pytest.mark.parametrize("group,field", [(3, 1), (3, 2), (2, 1)])
def test_run_fmunu_and_profiles(tmp_path, group, field):
    """FMUNU / F0MU with PL_LEVEL 3 and action profiles: the CPU re-check of
    F passes, the results file carries the FMUNU line, the 16 F columns
    (|F| = root of the sum of squares of the planes) and the two
    profile sections with one entry per slice"""
    dims = (4, 6, 4, 6)
    cfg = Q.default_config(group=group, size=dims, precision=1, start=Q.START_HOT, prng=Q.PRNG_PHILOX,
                           beta=5.8 if group == 3 else 2.3, row_align=64, n_or=1)
    opts = Q.default_run_options(iter=4, niter=1, nav=2, pl_level=3, quiet=1, fmunu=field, get_actions_diff=1,
                                 fmunu_index1=4 if group == 3 else 1, output_path=str(tmp_path) + "/",
                                 prefix="su%d-" % group)
    res = Q.run(cfg, opts)
    assert res.verification_passed == 1
    i1, i2 = (4, 8) if group == 3 else (1, 2)
    last = np.array(res.fmunu_gpu_last[:])
    assert np.allclose(last, np.array(res.fmunu_cpu_last[:]), rtol=1e-10, atol=1e-13)
    for g in range(2):
        for ri in range(2):
            assert abs(last[12 + 2 * g + ri] - np.sqrt(sum(last[6 * g + 2 * p + ri] ** 2 for p in range(3)))) < 1e-15
    text = open(res.results_file.decode()).read()
    assert (" FMUNU(%d, %d)" if field == 1 else " F0MU(%d, %d)") % (i1, i2) in text
    name = ("Fmunu_xy_%d_re" if field == 1 else "Fmunu_xt_%d_re") % i1
    assert " Mean %-20s:" % name in text
    assert "Differentiated Polyakov loop data (#, PL, PL_im, PL_variance, PL_im_variance):" in text
    assert "Differentiated S data (#, S_total, S_variance):" in text
    lines = text.split("\n")
    for a, tag in enumerate(("X", "Y", "Z")):
        rows = [l for l in lines if l.startswith(tag + "              ")]
        assert len(rows) == 2 and all(len(r.split()) == 1 + dims[a] for r in rows), tag
    pl_rows = [l for l in lines if l.startswith("PL             ")]
    assert len(pl_rows) == 3 and all(len(r.split()) == 1 + dims[a] for a, r in enumerate(pl_rows))
    # the CPU lattice variance of each F projection on the final field
    # (SU(2): the generator projections are real, their Im columns vanish)
    varnc = [float(l.split(":")[1]) for l in lines if l.startswith(" CPU l.varnc")]
    assert len(varnc) == 12 and all(v >= 0 for v in varnc), varnc
    assert all(v > 0 for v in (varnc if group == 3 else varnc[0::2])), varnc
    if group == 2:
        assert all(v == 0 for v in varnc[1::2]), varnc
    rows = [l for l in lines if l[:5].strip().isdigit()]
    assert len(rows) == 4
    # #, plaquettes 3, actions 3, Polyakov 2, P2/P4 2, F_munu 16
    vals = rows[-1].split()
    assert len(vals) == 1 + 3 + 3 + 2 + 2 + 16
    assert np.allclose([float(v) for v in vals[-16:]], last, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("group,precision", [(3, 0), (3, 1), (2, 1)])
def test_field_check_counts_broken_links(group, precision):
    """qg_field_check: a hot field passes; one NaN or one stretched link is
    counted once, and Gram-Schmidt does not hide a NaN"""
    cfg = Q.default_config(group=group, size=(4, 4, 4, 6), precision=precision, start=Q.START_HOT,
                           prng=Q.PRNG_PHILOX, beta=5.8, n_or=1)
    L = Q.Lattice(cfg)
    L.seed()
    L.init(Q.START_HOT)
    L.sweep(2)
    assert L.field_check() == 0
    good = L.download()
    t = good.copy()
    t[5] = np.nan                                    # plane 0 (direction x), site 1, one real
    L.upload(t)
    assert L.field_check() == 1
    L.reunitarize(True)
    assert L.field_check() == 1
    t = good.copy()
    P = 12 if group == 3 else 4
    rows = t.size // (P * 4)
    t.reshape(P, rows, 4)[2, 7, :] *= 1.01           # direction z at site 7: row norms off by ~2 %
    L.upload(t)
    assert L.field_check() == 1
    L.close()


def test_run_resumed_from_a_state_file_with_a_nan_link_reports_it(tmp_path):
    """host-side fault injection: a .qcg whose link table carries one NaN,
    resumed with INIT = 0, ends with QG_ERR_NUMERIC from the final field
    check instead of returning averages"""
    base = dict(group=3, size=(4, 4, 4, 4), precision=0, start=Q.START_COLD, prng=Q.PRNG_PHILOX, beta=5.9,
                row_align=64, n_or=1, reunit_every=2)
    good = str(tmp_path / "good.qcg")
    Q.run(Q.default_config(**base), Q.default_run_options(iter=2, niter=1, nav=1, quiet=1, write_results=0,
                                                          verify=0, save_state=1, state_out=good))
    cfg, st, ser, table = Q.read_state_file(good)
    table = table.copy()
    table[40] = np.nan
    bad = str(tmp_path / "bad.qcg")
    st.iter = 4
    Q.write_state_file(bad, cfg, st, table, ser)
    with pytest.raises(Q.QGError) as e:
        Q.run(Q.default_config(), Q.default_run_options(init=0, state_file=bad, quiet=1, write_results=0,
                                                        verify=0, save_state=0))
    assert "not finite or not in SU(N)" in str(e.value)


def test_profile_table_leaves_the_run_unchanged(tmp_path):
    """PROFILE = 1: every kernel class gets a time per launch, and the run's
    final table and series equal those of the same run without it (the
    timing launches work on a copy that is restored)"""
    base = dict(group=3, size=(4, 4, 4, 8), precision=0, start=Q.START_HOT, prng=Q.PRNG_PHILOX, beta=5.9,
                row_align=64, n_or=1, reunit_every=2, wilson_r=2, wilson_t=2)
    outs = []
    for profile in (0, 1):
        path = str(tmp_path / ("p%d.qcg" % profile))
        res = Q.run(Q.default_config(**base), Q.default_run_options(iter=3, niter=2, nav=2, get_wilson=1, quiet=1,
                                                                    write_results=0, verify=0, save_state=1,
                                                                    state_out=path, profile=profile))
        outs.append((res, Q.read_state_file(path)))
    assert all(x == 0.0 for x in outs[0][0].kernel_ms)
    assert all(x > 0.0 for x in outs[1][0].kernel_ms)
    assert np.array_equal(outs[0][1][3], outs[1][1][3])
    for k in outs[0][1][2]:
        assert np.array_equal(outs[0][1][2][k], outs[1][1][2][k]), k
    L = Q.Lattice(Q.default_config(**base))
    L.seed()
    L.init(Q.START_HOT)
    before = L.download()
    t = L.profile_kernels(reps=3)
    assert set(t) == set(Q.KERNEL_NAMES) and all(m > 0 for m, _ in t.values())
    assert np.array_equal(L.download(), before) and L.info().phase_counter == 0
    L.close()


@pytest.mark.parametrize("group,beta", [(3, 5.9), (2, 2.3)])
def test_run_results_file_follows_the_reference_writer(tmp_path, group, beta):
    """qg_run with the settings of the reference's own results file
    (tests/golden/reference_results_su{3,2}.txt, written by its CPU_RUN
    main()): the file it writes has the reference's layout line by line
    (test_results_file.py's comparison), the cold start's row 0 equals the
    reference's, and the verification line reports the CPU re-check"""
    import re
    import test_results_file as TR
    ref = open(os.path.join(TR.GOLDEN, "reference_results_su%d.txt" % group)).read().split("\n")
    cfg = Q.default_config(group=group, size=(4, 4, 4, 6), precision=1, start=Q.START_COLD, prng=Q.PRNG_RANLUX,
                           beta=beta, randseries=54, nhit=10, ranlux_nskip=223)
    opts = Q.default_run_options(iter=4, niter=2, nav=2, pl_level=0, get_wilson=0, fmunu=0, get_plaquettes=1,
                                 get_actions=1, quiet=1, output_path=str(tmp_path) + "/", prefix="su%d-" % group)
    res = Q.run(cfg, opts)
    got = open(res.results_file.decode()).read().split("\n")
    pats = TR.gpu_build_layout(ref)
    assert len(got) == len(pats)
    for i, (g, p) in enumerate(zip(got, pats)):
        assert re.fullmatch(p, g), (i + 1, g, p)
    row0 = [l for l in got if l[:5].strip() == "0"][0]
    assert row0.split() == [l for l in ref if l[:5].strip() == "0"][0].split()
    assert " *** Verification successfully passed! *" in "\n".join(got)
