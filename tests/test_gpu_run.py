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
