"""Regenerates tests/golden/stat_parity.json: long-run ensemble averages of
the plaquette from the reference's own sequential heatbath (SU(N)/suncpp,
the -D CPU_RUN build of vadimdi/QCDGPU), built from its sources by
oracle/build_ref.sh into oracle/_ref/ref_cpurun.

For each case: independent chains (RANDSERIES 101, 102, ...) from a cold
start (the reference's CPU hot start leaves the links zero), `therm`
sweeps dropped, then `sweeps` measured sweeps.  Per chain the mean of the
total plaquette (Re Tr, range [-N, N]) and its error sqrt(2 tau_int var / n)
with tau_int from the Madras-Sokal automatic window (c = 6); the case's
mean is the average over chains and its error the combined chain errors.

Usage: python tests/golden/make_stat_golden.py   (needs oracle/_ref built;
about five minutes on 8 cores)
"""
import json
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
EXE = os.path.join(ROOT, "oracle", "_ref", "ref_cpurun")

CASES = [
    {"name": "su3_4x4_b5.7", "group": 3, "dims": [4, 4, 4, 4], "beta": 5.7, "chains": 8, "therm": 500,
     "sweeps": 6000},
    {"name": "su2_4x4_b2.3", "group": 2, "dims": [4, 4, 4, 4], "beta": 2.3, "chains": 8, "therm": 500,
     "sweeps": 12000},
    # the lattice and coupling of the SU(2) run configuration (8^4, beta = 2.3), cold start
    {"name": "su2_8x4_b2.3", "group": 2, "dims": [8, 8, 8, 8], "beta": 2.3, "chains": 8, "therm": 500,
     "sweeps": 5000},
    {"name": "su3_8x4_b5.7", "group": 3, "dims": [8, 8, 8, 8], "beta": 5.7, "chains": 8, "therm": 300,
     "sweeps": 3000},
]


def tau_int(x, c=6.0):
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    d = x - x.mean()
    c0 = np.dot(d, d) / n
    t = 0.5
    for w in range(1, n):
        t += np.dot(d[:-w], d[w:]) / n / c0
        if w >= c * t:
            return t
    return t


def chain(case, series):
    args = [EXE, "plaq", str(case["group"])] + [str(d) for d in case["dims"]] + \
        [repr(case["beta"]), "1", str(series), str(case["therm"] + case["sweeps"])]
    tot = []
    for line in subprocess.check_output(args).decode().split("\n"):
        if line.strip():
            s, sp, tp, t = line.split()
            if int(s) > case["therm"]:
                tot.append(float(t))
    x = np.array(tot)
    tau = tau_int(x)
    return float(x.mean()), float(np.sqrt(2 * tau * x.var() / len(x))), float(tau)


def main():
    out = {"source": "reference CPU_RUN heatbath (SU(N)/suncpp), RANLUX3, NHIT=10, cold start",
           "observable": "total plaquette, mean Re Tr over sites and planes / 3 (range [-N, N])", "cases": []}
    with ThreadPoolExecutor(8) as ex:
        for case in CASES:
            res = list(ex.map(lambda k: chain(case, 101 + k), range(case["chains"])))
            means = np.array([r[0] for r in res])
            errs = np.array([r[1] for r in res])
            c = dict(case)
            c["mean"] = float(means.mean())
            c["error"] = float(np.sqrt(np.sum(errs ** 2)) / len(errs))
            c["tau_int"] = [r[2] for r in res]
            c["chain_means"] = means.tolist()
            out["cases"].append(c)
            print(c["name"], c["mean"], c["error"])
    with open(os.path.join(HERE, "stat_parity.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
