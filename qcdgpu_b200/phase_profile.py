"""Launches the sweep's phase kernels on one lattice, for a profiler.

  python -m qcdgpu_b200.phase_profile [--size 32] [--precision 0] [--group 3]
                                      [--prng philox|ranlux] [--warm 2] [--phases 1]
                                      [--shape S] [--kernel-table REPS]

Cold start, `warm` heatbath sweeps (8 heatbath phase launches each, so a
profiler skips 8*warm + 1 kernel launches to reach the measured ones), then
`phases` heatbath phase launches followed by `phases` overrelaxation phase
launches (odd X first), then the --measure measurements (each a kernel
and its reduction), then a synchronise.  --shape pins the launch shape of
both kinds (0 .. QG_TUNE_SHAPES-1) before the warm-up sweeps.
"""
import argparse

import qcdgpu_b200 as Q


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=32)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--group", type=int, default=3)
    ap.add_argument("--prng", default="philox", choices=["philox", "ranlux"])
    ap.add_argument("--warm", type=int, default=2)
    ap.add_argument("--phases", type=int, default=1)
    ap.add_argument("--shape", type=int, default=0)
    ap.add_argument("--kernel-table", type=int, default=0,
                    help="after the rest, print qg_profile_kernels' per-launch times (this many launches per class)")
    ap.add_argument("--measure", default="",
                    help="comma list run after the phases: wilson_all (8x8, FP32 products), "
                         "wilson_all64 (FP64 products), fmunu, action_profile, polyakov_profile, plaquette")
    a = ap.parse_args()
    cfg = Q.default_config(group=a.group, size=a.size, precision=a.precision, start=Q.START_COLD,
                           prng=Q.PRNG_PHILOX if a.prng == "philox" else Q.PRNG_RANLUX, beta=6.0, n_or=0,
                           reunit_every=0)
    L = Q.Lattice(cfg)
    L.set_shapes(a.shape, a.shape)
    L.seed()
    L.init()
    L.sweep(a.warm)
    for k in range(a.phases):
        if a.prng == "ranlux":
            L.produce()
        L.phase(1, k % 4, Q.HEATBATH)
    for k in range(a.phases):
        L.phase(1, k % 4, Q.OVERRELAX)
    for m in [x for x in a.measure.split(",") if x]:
        if m == "wilson_all":
            L.wilson_all(8, 8, fp64_products=False)
        elif m == "wilson_all64":
            L.wilson_all(8, 8, fp64_products=True)
        elif m == "fmunu":
            L.fmunu(Q.FMUNU_H)
        elif m == "action_profile":
            L.action_profile(0)
        elif m == "polyakov_profile":
            L.polyakov_profile(0)
        elif m == "plaquette":
            L.plaquette_sums()
        else:
            raise SystemExit("unknown measurement " + m)
    L.sync()
    print("plaquette", L.plaquette())
    if a.kernel_table:
        for name, (m, sd) in L.profile_kernels(a.kernel_table).items():
            print("%-22s %9.4f ms +- %.4f" % (name, m, sd))


if __name__ == "__main__":
    main()
