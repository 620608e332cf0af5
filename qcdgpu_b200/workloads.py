"""The named run configurations on one GPU, with the observables and
numbers each one reports.

  python -m qcdgpu_b200.workloads --config c1|c2|c2b|c5 [--sweeps N] [--therm N]

c1  SU(2) 8^4 beta=2.3, Haar hot start, sweep = 1 heatbath + 2
    overrelaxation, 200 + 1000 sweeps, plaquette and Polyakov loop every
    sweep, FP64 links.
c2  SU(3) 32^4 beta=6.0, cold start, Cabibbo-Marinari heatbath + 4
    overrelaxation, FP32 links, FP64 reductions and FP64 reunitarisation
    every 10 sweeps -- and the same chain (same seed) with all-FP64 links:
    the observables of both and their difference in units of the combined
    statistical error, plus the short-time divergence of the two chains
    from the same start (max |dU| and plaquette difference after 1, 2, 5,
    10 sweeps).
c2b the same at 24^3 x 6, beta = 5.9.
c5  SU(3) 64^4 beta=6.2, FP32 links, heatbath + 4 overrelaxation,
    plaquette, Polyakov loop and all planar Wilson loops up to 8 x 8
    (FP32 products, FP64 sums) every 10 sweeps; sweep throughput with and without the measurements
    and the overrelaxation phase's fraction of the HBM roofline.

Synthetic data: the lattices start cold or from a seeded hot start (no
configuration files).  Timings are CUDA events on the context's stream.
Prints one JSON line.
"""
import argparse
import json
import os

import numpy as np
import torch

import qcdgpu_b200 as Q

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def lattice(group, size, precision, beta, start, n_or, seed=54, reunit_fp64=1):
    L = Q.Lattice(Q.default_config(group=group, size=size, precision=precision, start=start, prng=Q.PRNG_PHILOX,
                                   beta=beta, randseries=seed, n_or=n_or, reunit_every=10, reunit_fp64=reunit_fp64))
    L.seed(seed)
    L.init()
    return L


def timed(L, fn):
    s = torch.cuda.ExternalStream(L.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    L.sync()
    e0.record(s)
    fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1)


def series(L, n, every=1):
    """n measurements, `every` sweeps apart: plaquette (mean Re Tr per
    plaquette, range [-N, N]), Re P and |P| (per spatial site, / N)"""
    V = float(np.prod(list(L.cfg.size)))
    nsp = float(L.cfg.size[0] * L.cfg.size[1] * L.cfg.size[2])
    N = L.cfg.group
    plq, pre, pab = np.zeros(n), np.zeros(n), np.zeros(n)
    for i in range(n):
        L.sweep(every)
        sp, tp = L.plaquette_sums()
        plq[i] = (sp + tp) / (6.0 * V)
        p = L.polyakov_sums()
        pre[i] = p[0] / (nsp * N)
        pab[i] = np.hypot(p[0], p[1]) / (nsp * N)
    return plq, pre, pab


def stat(x):
    tau, _ = Q.tau_int(x)
    return {"mean": float(x.mean()), "error": float(np.sqrt(2 * tau * x.var() / len(x))), "tau_int": tau}


def run_c1(a):
    L = lattice(2, (8, 8, 8, 8), 1, 2.3, Q.START_HAAR, 2)
    L.sweep(a.therm or 200)
    n = a.sweeps or 1000
    plq, pre, pab = series(L, n)
    t = timed(L, lambda: L.sweep(100)) / 100
    V = 8 ** 4
    return {"config": "c1", "workload": "SU(2) 8^4 beta=2.3, Haar start, 1 HB + 2 OR, FP64",
            "sweeps": n, "plaquette": stat(plq), "polyakov_re": stat(pre), "polyakov_abs": stat(pab),
            "ms_per_sweep": t, "link_updates_per_s": 4.0 * V * 3 / (t * 1e-3)}


def run_c2(a, size, beta, label):
    n = a.sweeps or 400
    therm = a.therm if a.therm is not None else 200
    out = {"config": label, "workload": "SU(3) %s beta=%g, cold start, 1 HB + 4 OR; FP32 links vs all-FP64"
                                        % ("x".join(map(str, size)), beta), "sweeps": n, "therm": therm}
    V = float(np.prod(size))
    # short-time divergence of the two chains from the same (cold) start
    L32 = lattice(3, size, 0, beta, Q.START_COLD, 4)
    L64 = lattice(3, size, 1, beta, Q.START_COLD, 4, reunit_fp64=1)
    div, done = [], 0
    for k in (1, 2, 5, 10):
        L32.sweep(k - done)
        L64.sweep(k - done)
        done = k
        u32, u64 = L32.download().astype(np.float64), L64.download()
        p32, p64 = sum(L32.plaquette_sums()) / (6 * V), sum(L64.plaquette_sums()) / (6 * V)
        div.append({"sweeps": k, "max_abs_dU": float(np.max(np.abs(u32 - u64))), "plaquette_diff": p32 - p64})
    out["divergence_from_same_start"] = div
    res = {}
    for name, L in (("fp32", L32), ("fp64", L64)):
        L.sweep(therm)
        ms = timed(L, lambda: L.sweep(20)) / 20
        plq, pre, pab = series(L, n)
        res[name] = {"plaquette": stat(plq), "polyakov_re": stat(pre), "polyakov_abs": stat(pab),
                     "ms_per_sweep": ms, "link_updates_per_s": 4.0 * V * 5 / (ms * 1e-3)}
        L.close()
    out.update(res)
    out["fp32_minus_fp64"] = {
        k: {"diff": res["fp32"][k]["mean"] - res["fp64"][k]["mean"],
            "sigma": float(np.hypot(res["fp32"][k]["error"], res["fp64"][k]["error"]))}
        for k in ("plaquette", "polyakov_re", "polyakov_abs")}
    return out


def run_c5(a):
    size = (64, 64, 64, 64)
    V = float(64 ** 4)
    L = lattice(3, size, 0, 6.2, Q.START_COLD, 4)
    L.sweep(a.therm if a.therm is not None else 20)
    tune = L.tune(reps=4)
    n = a.sweeps or 100
    ms_sweep = timed(L, lambda: L.sweep(10)) / 10
    meas = []

    def run():
        for k in range(n // 10):
            L.sweep(10)
            meas.append((L.plaquette_sums(), L.polyakov_sums(), L.wilson_all(8, 8, fp64_products=False)))
    ms_total = timed(L, run)
    ms_wilson = timed(L, lambda: L.wilson_all(8, 8, fp64_products=False))
    ms_wilson64 = timed(L, lambda: L.wilson_all(8, 8, fp64_products=True))
    peak, kind = hbm_peak()
    hb, orr = L.shapes()
    or_ms = tune[orr][1]
    alg = 4.5 * V * 48
    w = np.array([m[2] for m in meas]) / (3.0 * V)
    plq = np.array([sum(m[0]) / (6.0 * V) for m in meas])
    return {"config": "c5", "workload": "SU(3) 64^4 beta=6.2, FP32, 1 HB + 4 OR, measurements every 10 sweeps",
            "field_bytes": L.info().link_bytes, "sweeps": n, "ms_per_sweep": ms_sweep,
            "link_updates_per_s": 4.0 * V * 5 / (ms_sweep * 1e-3),
            "ms_per_sweep_with_measurements": ms_total / n,
            "link_updates_per_s_with_measurements": 4.0 * V * 5 * n / (ms_total * 1e-3),
            "ms_wilson_all_8x8": ms_wilson, "ms_wilson_all_8x8_fp64_products": ms_wilson64,
            "roofline": {"kernel": "overrelaxation phase", "achieved_gbs": alg / (or_ms * 1e-3) / 1e9,
                         "peak_gbs": peak, "peak_kind": kind, "frac": alg / (or_ms * 1e-3) / 1e9 / peak,
                         "ms_per_launch": or_ms},
            "plaquette_last": float(plq[-1]), "wilson_loops_last": w[-1].tolist()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", required=True, choices=["c1", "c2", "c2b", "c5"])
    ap.add_argument("--sweeps", type=int, default=None)
    ap.add_argument("--therm", type=int, default=None)
    a = ap.parse_args()
    if a.config == "c1":
        out = run_c1(a)
    elif a.config == "c2":
        out = run_c2(a, (32, 32, 32, 32), 6.0, "c2")
    elif a.config == "c2b":
        out = run_c2(a, (24, 24, 24, 6), 5.9, "c2b")
    else:
        out = run_c5(a)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
