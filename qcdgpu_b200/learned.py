"""Learned-proposal Metropolis against plain heatbath on one GPU.

  python -m qcdgpu_b200.learned [--size 16] [--beta 5.7] [--train-configs 2000]
                                [--steps-per-config 2] [--lr 2e-3] [--eps-max 1.5]
                                [--chain-sweeps 2000] [--nhits 1,4,8] [--seed 7]

SU(3) Wilson action, FP32 links, Philox stream.  After cold start and
heatbath thermalisation:
  1. the constant step (the proposal without a network) is scanned for the
     largest expected squared jump distance (ESJD) per proposal;
  2. the network starts from that step (output bias) and is trained with
     Adam on heatbath-generated configurations: one heatbath sweep, then
     `steps-per-config` gradient steps on its links, `train-configs` times;
  3. trained and constant proposals are compared on the same fresh
     heatbath configurations (ESJD, acceptance; paired difference);
  4. chains from the same thermalised configuration -- heatbath, and
     constant-step and learned Metropolis with each hit count in `nhits`
     (hits per SU(2) subgroup and link; the staple, its features and the
     network are evaluated once per link whatever the count) -- are run
     `chain-sweeps` sweeps with plaquette and Polyakov loop measured every
     sweep; reported: acceptance, mean plaquette with its tau_int-corrected
     error, tau_int of the plaquette and of Re P, sweeps/s of the update
     alone (CUDA events) and decorrelated configurations/s
     = sweeps/s / (2 tau_int) for each of the two observables.
Prints one JSON line.
"""
import argparse
import json
import time

import numpy as np
import torch

import qcdgpu_b200 as Q


def make(size, beta, seed):
    cfg = Q.default_config(group=3, size=size, precision=0, start=Q.START_COLD, prng=Q.PRNG_PHILOX, beta=beta,
                           randseries=seed, n_or=0, reunit_every=10, reunit_fp64=1, row_align=64)
    L = Q.Lattice(cfg)
    L.seed(seed)
    L.init()
    return L


def esjd_all_phases(L):
    """mean (ESJD, acceptance) over the 8 phases of the current field"""
    e, a = [], []
    for par in (1, 0):
        for mu in range(4):
            _, st = L.net_grad(par, mu)
            e.append(st[1] / 3.0)           # per proposal
            a.append(st[2])
    return float(np.mean(e)), float(np.mean(a))


def timed(L, fn, n):
    s = torch.cuda.ExternalStream(L.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    L.sync()
    e0.record(s)
    fn(n)
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / n


def chain(L, update, n, V, nsp):
    plq, pre = np.zeros(n), np.zeros(n)
    for i in range(n):
        update(1)
        sp, tp = L.plaquette_sums()
        plq[i] = (sp + tp) / (6.0 * V)
        pre[i] = L.polyakov_sums()[0] / (3.0 * nsp)
    tp_, _ = Q.tau_int(plq)
    tP, _ = Q.tau_int(pre)
    err = float(np.sqrt(2 * tp_ * plq.var() / n))
    return {"plaquette": float(plq.mean()), "plaquette_error": err, "tau_int_plaquette": tp_,
            "tau_int_polyakov": tP, "polyakov_abs": float(np.abs(pre).mean())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=16)
    ap.add_argument("--beta", type=float, default=5.7)
    ap.add_argument("--train-configs", type=int, default=2000)
    ap.add_argument("--steps-per-config", type=int, default=2)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--eps-max", type=float, default=1.5)
    ap.add_argument("--chain-sweeps", type=int, default=2000)
    ap.add_argument("--therm", type=int, default=200)
    ap.add_argument("--nhits", default="1,4,8")
    ap.add_argument("--eval-configs", type=int, default=16)
    ap.add_argument("--seed", type=int, default=7)
    a = ap.parse_args()
    size = (a.size,) * 4
    V = float(a.size ** 4)
    nsp = float(a.size ** 3)
    t0 = time.time()
    L = make(size, a.beta, a.seed)
    L.sweep(a.therm)
    therm_state = L.download()
    # 1. constant step scan
    grid = [0.15, 0.25, 0.35, 0.45, 0.55, 0.7, 0.85, 1.0]
    scan = []
    for eps in grid:
        L.net_set(Q.net_constant(eps, a.eps_max), a.eps_max)
        scan.append(esjd_all_phases(L)[0])
    best = grid[int(np.argmax(scan))]
    const_w = Q.net_constant(best, a.eps_max)
    # 2. training on heatbath configurations
    r = best / a.eps_max
    w0 = Q.net_init(seed=a.seed, out_bias=float(np.log(r / (1 - r))))
    L.net_set(w0, a.eps_max)
    hist = []
    for k in range(a.train_configs):
        L.sweep(1)
        st = L.net_train(a.steps_per_config, a.lr)
        if k % max(1, a.train_configs // 20) == 0:
            hist.append(st[1] / 3.0)
    trained_w, _ = L.net_get()
    # 3. paired comparison on fresh heatbath configurations
    d_esjd, e_tr, e_co, a_tr, a_co = [], [], [], [], []
    for k in range(a.eval_configs):
        L.sweep(2)
        L.net_set(trained_w, a.eps_max)
        et, at = esjd_all_phases(L)
        L.net_set(const_w, a.eps_max)
        ec, ac = esjd_all_phases(L)
        e_tr.append(et); e_co.append(ec); a_tr.append(at); a_co.append(ac); d_esjd.append(et - ec)
    gain = float(np.mean(e_tr) / np.mean(e_co) - 1.0)
    gain_err = float(np.std(d_esjd) / np.sqrt(len(d_esjd)) / np.mean(e_co))
    # 4. chains from the same thermalised configuration
    nhits = [int(v) for v in a.nhits.split(",")]
    out = {"workload": "SU(3) %d^4 beta=%g, FP32 links; learned vs constant-step Metropolis vs heatbath"
                       % (a.size, a.beta),
           "train_configs": a.train_configs, "steps_per_config": a.steps_per_config, "lr": a.lr,
           "eps_max": a.eps_max, "nhits": nhits, "constant_step_scan": dict(zip(map(str, grid), scan)),
           "best_constant_step": best, "training_esjd_history": hist,
           "esjd_trained": float(np.mean(e_tr)), "esjd_constant": float(np.mean(e_co)),
           "acceptance_trained": float(np.mean(a_tr)), "acceptance_constant": float(np.mean(a_co)),
           "esjd_gain": gain, "esjd_gain_error": gain_err, "chains": {}}
    runs = [("heatbath", None, 0)] + [(kind + "_nhit%d" % h, w, h) for h in nhits
                                      for kind, w in (("constant_step", const_w), ("learned", trained_w))]
    for name, w, nh in runs:
        L.upload(therm_state)
        if w is None:
            upd = L.sweep
        else:
            L.net_set(w, a.eps_max)
            upd = lambda n, nh=nh: L.mh_sweep(n, nh)   # noqa: E731
        ms = timed(L, upd, 50)
        L.mh_stats(reset=True) if w is not None else None
        res = chain(L, upd, a.chain_sweeps, V, nsp)
        if w is not None:
            res["acceptance"] = L.mh_stats()[0]
        res["ms_per_sweep"] = ms
        res["sweeps_per_s"] = 1000.0 / ms
        res["decorrelated_configs_per_s_polyakov"] = res["sweeps_per_s"] / (2.0 * res["tau_int_polyakov"])
        res["decorrelated_configs_per_s_plaquette"] = res["sweeps_per_s"] / (2.0 * res["tau_int_plaquette"])
        out["chains"][name] = res
    out["seconds"] = time.time() - t0
    print(json.dumps(out))


if __name__ == "__main__":
    main()
