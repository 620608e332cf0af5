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
    files = [f for f in os.listdir(str(tmp_path)) if f.startswith("su3-") and f.endswith(".txt")]
    assert len(files) == 1


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
    common = dict(niter=2, nav=3, pl_level=2, get_wilson=1, quiet=1, write_results=0, verify=0, save_state=1)
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
