"""The results file's layout against the reference's own writer.

tests/golden/reference_results_su{3,2}.txt are results files written by the
reference's main() (its CPU_RUN build, oracle/_ref/ref_qcdgpu; made by
tests/golden/make_results_golden.py) for SU(3) and SU(2) 4x4x4x6 cold
starts.  qg_write_results (what qg_run writes) is fed a run of the same
settings and must reproduce the file line by line: the same sections in
the same order, the same labels and column widths, numbers and times
masked.  Three differences between the reference's CPU_RUN build and its
GPU build (lattice_make_header and lattice_make_header2 in
SU(N)/suncl/suncl.cpp) are applied to the golden file before the
comparison, since this library follows the GPU build: the
"Sequential run on CPU" line is the two device lines ("Active <platform>
platform / device"), a "precision" line follows "nhitPar", and the
verification line follows the last-value block.  Labels the reference
prints as "(null)" (observables its CPU_RUN build does not name) match any
label.
"""
import os
import re

import numpy as np
import pytest

import qcdgpu_b200 as Q

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
NUM = re.compile(r"[-+]?\d+\.\d+e[-+]\d+|[-+]?\d+")


def line_pattern(line):
    """regex for a reference line: numbers -> any number, "(null)" -> any
    label, the title's version and build tag -> any, times -> any"""
    if line.startswith(" Start time") or line.startswith(" Finish time"):
        return re.escape(line[:27]) + ".*"
    if line.startswith(" GPU SU("):
        return re.escape(line[:20]) + r" \S+ \(.*\)"
    out, pos = "", 0
    for m in re.finditer(r"\(null\)\s*|[-+]?\d+\.\d+e[-+]\d+|[-+]?\d+", line):
        out += re.escape(line[pos:m.start()])
        tok = m.group(0)
        if tok.startswith("(null)"):
            # the label is left-justified in a field of len(tok) characters
            out += r"\S+ *" if len(tok) > 6 else r"\S+"
        else:
            out += r"[-+ ]?\d+(\.\d+e[-+]\d+)?"
        pos = m.end()
    return out + re.escape(line[pos:])


def gpu_build_layout(lines):
    """the reference's CPU_RUN file as its GPU build lays it out"""
    out = []
    last_gpu = max(i for i, l in enumerate(lines) if l.startswith(" GPU last"))
    for i, l in enumerate(lines):
        if l.strip() == "Sequential run on  CPU":
            out += [re.escape(" Active ") + r"\S+" + re.escape(" platform     : ") + ".*",
                    re.escape(" Active ") + r"\S+" + re.escape(" device       : ") + ".*"]
            continue
        out.append(line_pattern(l))
        if l.startswith(" nhitPar"):
            out.append(re.escape(" precision                   : ") + "(single|double)")
        if i == last_gpu:
            out.append(r" (\*\*\* Verification successfully passed! \*+|--- Verification failed! -+)")
    return out


@pytest.mark.parametrize("group,beta", [(3, 5.9), (2, 2.3)])
def test_results_file_follows_the_reference_writer(tmp_path, group, beta):
    ref = open(os.path.join(GOLDEN, "reference_results_su%d.txt" % group)).read().split("\n")
    cfg = Q.default_config(group=group, size=(4, 4, 4, 6), precision=1, start=Q.START_COLD, prng=Q.PRNG_RANLUX,
                           beta=beta, randseries=54, nhit=10, ranlux_nskip=223)
    opts = Q.default_run_options(iter=4, niter=2, nav=2, pl_level=0, get_wilson=0, fmunu=0, get_plaquettes=1,
                                 get_actions=1, output_path=str(tmp_path) + "/", prefix="su%d-" % group)
    res = Q.RunResult()
    rng = np.random.default_rng(group)
    series = rng.uniform(0.5, 3.0, (Q.OBS_COUNT, 4))
    res.verification_passed = 1
    for k in range(Q.OBS_COUNT):
        res.mean[k], res.variance[k] = float(series[k, 1:].mean()), float(series[k, 1:].var())
        res.gpu_last[k] = res.cpu_last[k] = float(series[k, -1])
    path = Q.write_results(cfg, opts, res, series, t_start=1700000000, t_end=1700000042,
                           platform="CUDA 12.9", device="NVIDIA B200")
    got = open(path).read().split("\n")
    pats = gpu_build_layout(ref)
    assert len(got) == len(pats), (len(got), len(pats))
    for i, (g, p) in enumerate(zip(got, pats)):
        assert re.fullmatch(p, g), "line %d:\n  got     %r\n  pattern %r" % (i + 1, g, p)
    # the data rows carry the series
    rows = [l for l in got if l[:5].strip().isdigit()]
    assert len(rows) == 4
    for i, r in enumerate(rows):
        v = [float(x) for x in r.split()[1:]]
        want = series[[Q.OBS_PLQ_SPAT, Q.OBS_PLQ_TEMP, Q.OBS_PLQ_TOTAL, Q.OBS_S_SPAT, Q.OBS_S_TEMP,
                       Q.OBS_S_TOTAL], i]
        assert np.allclose(v, want, rtol=1e-12)
    # what this library adds sits in the companion file
    stats = open(path[:-4] + "-stats.txt").read()
    assert "Tau_int S_total" in stats and "overrelaxation sweeps" in stats
    assert "Tau_int" not in open(path).read()


def test_results_file_name_is_the_reference_stamp(tmp_path):
    cfg = Q.default_config(group=3, size=(4, 4, 4, 4))
    opts = Q.default_run_options(iter=1, pl_level=0, output_path=str(tmp_path) + "/", prefix="su3-")
    import time
    t = 1700000042
    path = Q.write_results(cfg, opts, Q.RunResult(), np.zeros((Q.OBS_COUNT, 1)), t_start=t, t_end=t)
    c = time.ctime(t)
    assert os.path.basename(path) == "su3-%s-%s-%s-%s-%s-%s.txt" % (c[22:24], c[4:7], c[8:10], c[11:13], c[14:16],
                                                                    c[17:19])


def test_results_file_elapsed_time_past_a_day(tmp_path):
    """days:hours:minutes:seconds with the hours taken modulo 24 (the
    reference's formula keeps counting hours past the first day)"""
    cfg = Q.default_config(group=2, size=(4, 4, 4, 4))
    opts = Q.default_run_options(iter=1, pl_level=0, output_path=str(tmp_path) + "/", prefix="su2-")
    t0 = 1700000000
    path = Q.write_results(cfg, opts, Q.RunResult(), np.zeros((Q.OBS_COUNT, 1)), t_start=t0,
                           t_end=t0 + 2 * 86400 + 5 * 3600 + 7 * 60 + 9)
    line = [l for l in open(path) if l.startswith(" Elapsed time")][0]
    assert line.rstrip().endswith(": 2:05:07:09"), line
