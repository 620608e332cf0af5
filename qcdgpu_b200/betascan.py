"""Batched beta scan: many independent SU(3) ensembles with different
extents and couplings, one launch per phase over all of them (qg_batch),
the sweep and the measurement captured in one CUDA graph -- on one GPU or
spread over the GPUs of a node.

  python -m qcdgpu_b200.betascan [--ensembles 64] [--sweeps 500] [--n-or 4]
                                 [--measure-every 1] [--seed 54] [--shape -1] [--persistent]
  torchrun --nproc-per-node N -m qcdgpu_b200.betascan ...   (one rank per GPU)

Workload: N_t drawn from {4, 6, 8} and N_s from {16, 20, 24, 32} with a
fixed seed, beta = 5.5 + 0.7 i / (n - 1), cold start, FP32 links, FP64
reunitarisation every 10 sweeps, Philox stream (RANDSERIES 1000 + i).
The batched launch shapes are autotuned after the warm-up sweeps
(qg_batch_tune, fields restored) unless --shape pins one.

Several GPUs (the multi-GPU replica scheduler): the ensembles are
independent, so they are dealt to the ranks by cost (sites x updates per
sweep, largest first, each to the least-loaded rank; deterministic) and
each rank runs its share as one batch -- no collective on the data path.
An ensemble's chain depends only on its own RANDSERIES and the sweep count,
so the results do not depend on the split.  Rank 0 gathers the
per-ensemble results; the job's time is the slowest rank's device time
(CUDA events on each batch's stream, barrier before and after).

Prints one JSON line: link updates/s over all ensembles, the per-ensemble
mean plaquette of the second half of the run and the Polyakov-loop
modulus, in ensemble order.
"""
import argparse
import json

import numpy as np

def workload(n, seed):
    rng = np.random.default_rng(seed)
    nt = rng.choice([4, 6, 8], size=n)
    ns = rng.choice([16, 20, 24, 32], size=n)
    betas = 5.5 + 0.7 * np.arange(n) / max(n - 1, 1)
    return [((int(s), int(s), int(s), int(t)), float(b), 1000 + i) for i, (s, t, b) in enumerate(zip(ns, nt, betas))]


def ensemble_cost(e, n_or):
    """link updates of one sweep of ensemble e = (size, beta, randseries)"""
    return 4 * int(np.prod(e[0])) * (1 + n_or)


def partition(ens, world, n_or=4):
    """ensemble indices per rank: largest cost first, each to the rank with
    the least load so far (lowest rank on ties); each list ascending"""
    load = [0] * world
    shares = [[] for _ in range(world)]
    for k in sorted(range(len(ens)), key=lambda k: (-ensemble_cost(ens[k], n_or), k)):
        r = min(range(world), key=lambda r: (load[r], r))
        shares[r].append(k)
        load[r] += ensemble_cost(ens[k], n_or)
    return [sorted(x) for x in shares]


def run_share(ens, idx, a):
    """run ensembles ens[idx] as one batch on this rank's GPU; per-ensemble
    observables, updates and the device time of the timed sweeps"""
    import torch

    import qcdgpu_b200 as Q
    if not idx:
        return {"idx": [], "plaquette": [], "polyakov_abs": [], "updates": 0.0, "ms": 0.0, "sites": 0,
                "field_bytes": 0, "shapes": None}
    sub = [ens[k] for k in idx]
    cfg = Q.default_config(group=3, precision=0, prng=Q.PRNG_PHILOX, n_or=a.n_or, reunit_every=10, reunit_fp64=1,
                           nhit=10, row_align=64)
    nmeas = (a.sweeps + a.warmup) // a.measure_every + 1
    B = Q.Batch(cfg, sub, max_measurements=nmeas)
    if getattr(a, "plaquette_fp32", False):
        B.set_measure_products(True)                  # FP32 products and traces, FP64 sums
    B.init(Q.START_COLD)
    stream = torch.cuda.ExternalStream(B.stream())
    B.run(a.warmup, a.measure_every)                  # warm-up, untimed
    if getattr(a, "persistent", False):
        B.set_persistent(True)                        # one launch per half-sweep (same chains)
    if a.shape < 0:
        B.tune()                                      # fields restored: the chains are unchanged
    else:
        B.set_shape(a.shape)
    shapes = list(B.shapes())
    B.run(1, a.measure_every)                         # graph capture with the chosen shapes, untimed
    B.sync()
    if a.barrier is not None:
        a.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    B.run(a.sweeps, a.measure_every)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    info = B.info()
    ser = B.series()
    V = np.array([np.prod(s) for s, _, _ in sub], dtype=np.float64)
    nsp = np.array([s[0] * s[1] * s[2] for s, _, _ in sub], dtype=np.float64)
    half = ser[ser.shape[0] // 2:]
    plaq = (half[:, :, 0] + half[:, :, 1]) / (6 * V)          # mean Re Tr per plaquette, range [-3, 3]
    poly = np.hypot(half[:, :, 4], half[:, :, 5]) / (3 * nsp)
    B.close()
    return {"idx": list(idx), "plaquette": plaq.mean(axis=0).tolist(), "polyakov_abs": poly.mean(axis=0).tolist(),
            "updates": 4.0 * info["sites"] * (1 + a.n_or) * a.sweeps, "ms": ms, "sites": info["sites"],
            "field_bytes": info["field_bytes"], "shapes": shapes}


def merge(parts, n):
    """rank results -> job result: per-ensemble values in ensemble order,
    the job time = the slowest rank's, the whole-job update rate"""
    plaq, poly = [None] * n, [None] * n
    for p in parts:
        for j, k in enumerate(p["idx"]):
            plaq[k], poly[k] = p["plaquette"][j], p["polyakov_abs"][j]
    ms = max(p["ms"] for p in parts)
    updates = sum(p["updates"] for p in parts)
    return {"plaquette": plaq, "polyakov_abs": poly, "ms": ms, "updates": updates,
            "link_updates_per_s": updates / (ms * 1e-3) if ms > 0 else 0.0,
            "sites": sum(p["sites"] for p in parts), "field_bytes": sum(p["field_bytes"] for p in parts),
            "ranks": [{"ensembles": len(p["idx"]), "ms": p["ms"], "shapes": p.get("shapes")} for p in parts]}


def schedule(ens, a, dist, rank, world, runner=run_share):
    """this rank's share through `runner`, gathered on every rank, merged"""
    shares = partition(ens, world, a.n_or)
    mine = runner(ens, shares[rank], a)
    if dist is None:
        parts = [mine]
    else:
        parts = [None] * world
        dist.all_gather_object(parts, mine)
    return merge(parts, len(ens))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ensembles", type=int, default=64)
    ap.add_argument("--sweeps", type=int, default=500)
    ap.add_argument("--n-or", type=int, default=4)
    ap.add_argument("--measure-every", type=int, default=1)
    ap.add_argument("--seed", type=int, default=54)
    ap.add_argument("--shape", type=int, default=-1, help="batched launch shape; -1 = autotune (qg_batch_tune)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--persistent", action="store_true",
                    help="one persistent launch per half-sweep (grid barriers between directions)")
    ap.add_argument("--plaquette-fp32", action="store_true",
                    help="measure the plaquette with FP32 products (FP64 sums) instead of FP64 products")
    a = ap.parse_args()
    import torch

    from qcdgpu_b200 import replicas as RP
    rank, world, local = RP.dist_env()
    torch.cuda.set_device(local)
    dist = RP.init("nccl", 300, torch.device("cuda", local)) if world > 1 else None
    a.barrier = (lambda: RP.barrier(dist)) if dist is not None else None
    ens = workload(a.ensembles, a.seed)
    job = schedule(ens, a, dist, rank, world)
    RP.barrier(dist)
    RP.finish(dist)
    if rank != 0:
        return
    print(json.dumps({
        "workload": "beta scan, %d SU(3) ensembles, N_s in {16,20,24,32}, N_t in {4,6,8}, beta 5.5..6.2, "
                    "1 HB + %d OR per sweep, FP32 links" % (a.ensembles, a.n_or),
        "gpus": world, "sites": job["sites"], "field_bytes": job["field_bytes"], "sweeps": a.sweeps,
        "measure_every": a.measure_every, "plaquette_products": "fp32" if a.plaquette_fp32 else "fp64",
        "ms": job["ms"], "ms_per_sweep": job["ms"] / a.sweeps,
        "link_updates_per_s": job["link_updates_per_s"], "ranks": job["ranks"],
        "beta": [b for _, b, _ in ens], "extents": [list(s) for s, _, _ in ens],
        "plaquette": job["plaquette"], "polyakov_abs": job["polyakov_abs"]}))


if __name__ == "__main__":
    main()
