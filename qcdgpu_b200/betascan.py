"""Batched beta scan on one GPU (qg_batch): many independent SU(3)
ensembles with different extents and couplings, one launch per phase over
all of them, the sweep and the measurement captured in one CUDA graph.

  python -m qcdgpu_b200.betascan [--ensembles 64] [--sweeps 500] [--n-or 4]
                                 [--measure-every 1] [--seed 54] [--shape 4]

Workload: N_t drawn from {4, 6, 8} and N_s from {16, 20, 24, 32} with a
fixed seed, beta = 5.5 + 0.7 i / (n - 1), cold start, FP32 links, FP64
reunitarisation every 10 sweeps, Philox stream (RANDSERIES 1000 + i).  The
timed region (CUDA events on the batch's stream) covers all sweeps and
measurements.  Prints one JSON line: link updates/s over all ensembles,
the per-ensemble mean plaquette of the second half of the run, and the
Polyakov-loop modulus.
"""
import argparse
import json

import numpy as np
import torch

import qcdgpu_b200 as Q


def workload(n, seed):
    rng = np.random.default_rng(seed)
    nt = rng.choice([4, 6, 8], size=n)
    ns = rng.choice([16, 20, 24, 32], size=n)
    betas = 5.5 + 0.7 * np.arange(n) / max(n - 1, 1)
    return [((int(s), int(s), int(s), int(t)), float(b), 1000 + i) for i, (s, t, b) in enumerate(zip(ns, nt, betas))]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ensembles", type=int, default=64)
    ap.add_argument("--sweeps", type=int, default=500)
    ap.add_argument("--n-or", type=int, default=4)
    ap.add_argument("--measure-every", type=int, default=1)
    ap.add_argument("--seed", type=int, default=54)
    ap.add_argument("--shape", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args()
    ens = workload(a.ensembles, a.seed)
    cfg = Q.default_config(group=3, precision=0, prng=Q.PRNG_PHILOX, n_or=a.n_or, reunit_every=10, reunit_fp64=1,
                           nhit=10, row_align=64)
    nmeas = (a.sweeps + a.warmup) // a.measure_every + 1
    B = Q.Batch(cfg, ens, max_measurements=nmeas)
    B.set_shape(a.shape)
    B.init(Q.START_COLD)
    stream = torch.cuda.ExternalStream(B.stream())
    B.run(a.warmup, a.measure_every)                  # graph capture and warm-up, untimed
    B.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    B.run(a.sweeps, a.measure_every)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    info = B.info()
    ser = B.series()
    V = np.array([np.prod(s) for s, _, _ in ens], dtype=np.float64)
    nsp = np.array([s[0] * s[1] * s[2] for s, _, _ in ens], dtype=np.float64)
    half = ser[ser.shape[0] // 2:]
    plaq = (half[:, :, 0] + half[:, :, 1]) / (6 * V)          # mean Re Tr per plaquette, range [-3, 3]
    poly = np.hypot(half[:, :, 4], half[:, :, 5]) / (3 * nsp)
    updates = 4.0 * info["sites"] * (1 + a.n_or) * a.sweeps
    print(json.dumps({
        "workload": "beta scan, %d SU(3) ensembles, N_s in {16,20,24,32}, N_t in {4,6,8}, beta 5.5..6.2, "
                    "1 HB + %d OR per sweep, FP32 links" % (a.ensembles, a.n_or),
        "sites": info["sites"], "field_bytes": info["field_bytes"], "sweeps": a.sweeps,
        "measure_every": a.measure_every, "ms": ms, "ms_per_sweep": ms / a.sweeps,
        "link_updates_per_s": updates / (ms * 1e-3),
        "beta": [b for _, b, _ in ens], "extents": [list(s) for s, _, _ in ens],
        "plaquette": plaq.mean(axis=0).tolist(), "polyakov_abs": poly.mean(axis=0).tolist()}))
    B.close()


if __name__ == "__main__":
    main()
