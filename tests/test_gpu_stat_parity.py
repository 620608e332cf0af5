"""Long-run parity with the reference: the GPU chain's ensemble average of
the plaquette agrees with the reference's own sequential heatbath
(tests/golden/stat_parity.json, made by tests/golden/make_stat_golden.py
from the reference's CPU_RUN build) within 2 sigma, sigma combining both
errors of the mean with their integrated autocorrelation times
(qg_run's tau_int, Madras-Sokal window).  Overrelaxation sweeps change the
dynamics, not the distribution, so the HB + OR chains must agree too."""
import json
import os

import numpy as np
import pytest

import qcdgpu_b200 as Q

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "stat_parity.json")))
CASES = {c["name"]: c for c in GOLD["cases"]}


@pytest.mark.parametrize("name,precision,n_or,series", [
    ("su3_4x4_b5.7", 0, 0, 11), ("su3_4x4_b5.7", 0, 4, 12), ("su3_4x4_b5.7", 1, 0, 13),
    ("su2_4x4_b2.3", 1, 2, 14), ("su2_4x4_b2.3", 0, 0, 15),
    # SU(2) 8^4 beta=2.3 FP64, 1 HB + 2 OR: the SU(2) run configuration (cold start)
    ("su2_8x4_b2.3", 1, 2, 16), ("su2_8x4_b2.3", 0, 0, 17),
    ("su3_8x4_b5.7", 0, 4, 18), ("su3_8x4_b5.7", 1, 0, 19)])
def test_plaquette_average_agrees_with_reference_heatbath(name, precision, n_or, series):
    case = CASES[name]
    cfg = Q.default_config(group=case["group"], size=tuple(case["dims"]), precision=precision, start=Q.START_COLD,
                           prng=Q.PRNG_PHILOX, beta=case["beta"], randseries=series, n_or=n_or, reunit_every=1)
    sweeps = 30000 if case["dims"][0] == 4 else 15000
    opts = Q.default_run_options(iter=sweeps + 1, niter=1, nav=500, pl_level=0, get_actions=0, get_plaquettes=1,
                                 quiet=1, write_results=0, verify=0)
    res = Q.run(cfg, opts)
    k = Q.OBS_NAMES.index("Plq_total")
    m, e, tau = res.mean[k], res.error[k], res.tau_int[k]
    assert 0.5 <= tau < 50 and e > 0
    sigma = np.hypot(e, case["error"])
    z = (m - case["mean"]) / sigma
    print("%s prec=%d n_or=%d: %.6f +- %.6f (tau %.2f) vs reference %.6f +- %.6f, z = %.2f" %
          (name, precision, n_or, m, e, tau, case["mean"], case["error"], z))
    assert abs(z) <= 2.0
