"""Benchmark of the SU(3) checkerboard sweep on B200.

Workload (one "step" = one full sweep): SU(3) Wilson action, 32^4 lattice,
beta = 6.0, FP32 12-real compressed links, sweep = 1 Cabibbo-Marinari
heatbath + 4 overrelaxation sweeps, FP64 reunitarisation every 10 sweeps,
cold start thermalised for a few untimed sweeps.  Metric: link updates per
second (4V links x 5 updates per sweep), whole job.  The link field
(201 MB) is larger than the 126 MB L2, so no L2 flush is needed between
steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun): independent replicas, one lattice per GPU (distinct seed),
no collective on the data path; barrier + max-over-ranks device time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SIZE = 32
BETA = 6.0
N_OR = 4
REUNIT_EVERY = 10
METRIC = "link updates/s (SU(3) 32^4 beta=6.0 FP32, 1 HB + 4 OR sweep)"
UNIT = "link_updates/s"
LINK_BYTES = 48          # 12 FP32 reals per stored SU(3) link


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)   # about 2.7 s timed: a dozen clock samples
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--prng", default="philox", choices=["philox", "ranlux"])
    ap.add_argument("--size", type=int, default=SIZE)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shapes", default=None,
                    help="HB,OR launch shapes to pin instead of tuning (e.g. for a profiler run)")
    return ap.parse_args()



# ------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = tempfile.mktemp(prefix="qg_clocks_", suffix=".csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------ reference (CPU)
def ref_binary():
    return os.path.join(ROOT, "oracle", "_ref", "ref_cpurun")


def cpu_workers(size):
    ncpu = os.cpu_count() or 1
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError):
        avail = 8 << 30
    per = 4 * size ** 4 * 18 * 8 * 1.3         # the reference CPU path stores links as 18 doubles
    return max(1, min(ncpu, 64, int(0.5 * avail // per)))


def run_reference_phases(size, procs, warm, timed):
    """The reference's sequential heatbath (SU(N)/suncpp) in `procs`
    concurrent processes with distinct RANDSERIES; each does `warm` + `timed`
    phases (V/2 link updates each) and reports per-phase wall times."""
    cmd = [ref_binary(), "phases", "3", str(size), str(size), str(size), str(size), repr(BETA)]
    ps = [subprocess.Popen(cmd + [str(54 + i), str(warm), str(timed)], stdout=subprocess.PIPE, text=True)
          for i in range(procs)]
    times = []
    for p in ps:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("reference CPU path failed")
        times.append([float(x) for x in out.split()[1:]])
    return times


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline_line(size, seconds_target=15.0):
    if not os.path.exists(ref_binary()):
        return None
    one = run_reference_phases(size, 1, 0, 1)[0][0]   # one process alone: the per-core rate
    procs = cpu_workers(size)
    t = run_reference_phases(size, procs, 0, 1)
    per_phase = max(x[0] for x in t)
    n = max(1, min(8, int(seconds_target / max(per_phase, 1e-3))))
    t = run_reference_phases(size, procs, 0, n)
    wall = max(sum(x) for x in t)
    links = procs * n * (size ** 4 // 2)
    return {"value": links / wall, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": "reference CPU path (SU(N)/suncpp heatbath, RANLUX3, NHIT=10; it has no overrelaxation) on "
                      "SU(3) %d^4 beta=%.1f cold start: %d concurrent processes x %d phases of %d link updates, "
                      "%.1f s wall" % (size, BETA, procs, n, size ** 4 // 2, wall),
            "single_process": {"value": (size ** 4 // 2) / one, "unit": UNIT, "cores": 1,
                               "sample": "one process alone, one phase of %d link updates, %.2f s"
                                         % (size ** 4 // 2, one)},
            "cpu_model": cpu_model(), "host_cpus": os.cpu_count()}


def table_rows_fp64(table, size, rowsize):
    """an FP64 SU(3) reference-layout table (12 planes of rowsize float4s)
    -> the reference CPU path's stored rows per (site, direction): u1 u2 u3
    v1 v2 v3 as (re, im), site-major, direction fastest"""
    import numpy as np
    V = size ** 4
    t = table.reshape(12, rowsize, 4)[:, :V, :]
    p1, p2, p3 = t[0:4].transpose(1, 0, 2), t[4:8].transpose(1, 0, 2), t[8:12].transpose(1, 0, 2)
    return np.ascontiguousarray(np.stack([p1[..., 0], p2[..., 0], p1[..., 1], p2[..., 1], p1[..., 2], p2[..., 2],
                                          p3[..., 0], p3[..., 2], p3[..., 1], p3[..., 3], p1[..., 3], p2[..., 3]],
                                         axis=-1))


def like_for_like(Q, torch, size, seconds_target=10.0):
    """Heatbath-only sweeps in the reference's own arithmetic on both sides:
    SU(3) size^4 beta=6.0, FP64 links, RANLUX3 batches (one per phase, the
    reference's lattice_simulate cadence; generated on the GPU inside the
    timed sweeps), NHIT=10, Gram-Schmidt every sweep.  Ours: CUDA events
    around 10 sweeps after 20 thermalising ones.  The reference CPU path
    (SU(N)/suncpp, FP64, RANLUX3, NHIT=10): the same thermalised FP64
    configuration loaded into each of its concurrent processes, per-phase
    wall times."""
    cfg = Q.default_config(group=3, size=size, precision=1, start=Q.START_COLD, prng=Q.PRNG_RANLUX, beta=BETA,
                           nhit=10, ranlux_nskip=223, n_or=0, reunit_every=1, reunit_fp64=1, randseries=54,
                           prng_instances=16384)
    L = Q.Lattice(cfg)
    L.seed()
    L.init()
    L.sweep(20)
    s = torch.cuda.ExternalStream(L.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    L.sync()
    e0.record(s)
    L.sweep(10)
    e1.record(s)
    e1.synchronize()
    ms_sweep = e0.elapsed_time(e1) / 10
    V = size ** 4
    out = {"what": "heatbath-only sweeps in the reference's own arithmetic: SU(3) %d^4 beta=%.1f, FP64 links, RANLUX3 "
                   "batches generated for every phase, NHIT=10, Gram-Schmidt every sweep, thermalised start (20 "
                   "sweeps)" % (size, BETA),
           "ours": {"value": 4 * V / (ms_sweep / 1e3), "unit": UNIT, "ms_per_phase": ms_sweep / 8,
                    "how": "CUDA events around 10 sweeps (8 RANLUX batches + 8 heatbath phases + Gram-Schmidt each)"}}
    if os.path.exists(ref_binary()):
        rows = table_rows_fp64(L.download(), size, L.info().rowsize)
        with tempfile.TemporaryDirectory() as d:
            f = os.path.join(d, "thermalised.bin")
            rows.tofile(f)
            procs = cpu_workers(size)
            cmd = [ref_binary(), "phases_from", "3"] + [str(size)] * 4 + [repr(BETA)]
            ps = [subprocess.Popen(cmd + [str(54 + i), f, "0", "2"], stdout=subprocess.PIPE, text=True)
                  for i in range(procs)]
            times = []
            for p in ps:
                o, _ = p.communicate()
                if p.returncode != 0:
                    raise RuntimeError("reference CPU path failed")
                times.append([float(x) for x in o.split()[1:]])
        wall = max(sum(t) for t in times)
        out["reference"] = {"value": procs * 2 * (V // 2) / wall, "unit": UNIT, "cores": procs,
                            "ms_per_phase_per_process": 1e3 * wall / 2,
                            "how": "%d concurrent processes of the reference CPU path, each from the same thermalised "
                                   "configuration, 2 heatbath phases of %d link updates each" % (procs, V // 2)}
    L.close()
    return out


REF_MAX_STEPS = 60


def run_reference_arm(args):
    from qcdgpu_b200 import replicas as RP
    rank, world, _ = RP.dist_env()
    if not RP.reference_arm_runs_here(rank):
        return 0
    if not os.path.exists(ref_binary()):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_cpurun not built"}))
        return 0
    procs = cpu_workers(args.size)
    # one step = one heatbath phase per process, about 1.2 s of CPU work at
    # 32^4: the timed steps are capped so that the run stays within a few
    # minutes whatever --steps asks for (the rate does not depend on it)
    steps = min(args.steps, REF_MAX_STEPS)
    try:
        t = run_reference_phases(args.size, procs, args.warmup, steps)
    except (RuntimeError, OSError, ValueError) as e:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU path failed: %s" % e}))
        return 0
    step = [max(x[k] for x in t) for k in range(steps)]
    total = sum(step)
    links = procs * steps * (args.size ** 4 // 2)
    value = links / total
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "steps_requested": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (cold start)",
            "impl": "reference",
            "config": {"workload": "SU(3) %d^4 beta=%.1f, FP32 12-real links, 1 HB + %d OR per sweep, FP64 reunit "
                                   "every %d" % (args.size, BETA, N_OR, REUNIT_EVERY),
                       "lattice": [args.size] * 4,
                       "reference_work": "the reference CPU path has heatbath updates only (no overrelaxation, "
                                         "FP64 links): per step one heatbath phase of V/2 link updates in each "
                                         "process", "processes": procs},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
                             "sample": "%d concurrent processes of the reference CPU path, one phase each per step"
                                       % procs},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------ our arm
def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic():
    """Per-launch DRAM bytes of the phase kernels from the committed ncu
    summary (profiles/phase_traffic.json), scaled to this lattice."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "phase_traffic.json")))
        return d
    except (OSError, ValueError):
        return None


def run_ours(args):
    import torch
    import qcdgpu_b200 as Q

    from qcdgpu_b200 import replicas as RP

    rank, world, local = RP.dist_env()
    torch.cuda.set_device(local)
    dist = RP.init("nccl", 120, torch.device("cuda", local)) if world > 1 else None
    prng = Q.PRNG_PHILOX if args.prng == "philox" else Q.PRNG_RANLUX
    cfg = Q.default_config(group=3, size=args.size, precision=0, start=Q.START_COLD, prng=prng, beta=BETA,
                           n_or=N_OR, reunit_every=REUNIT_EVERY, reunit_fp64=1, randseries=RP.replica_seed(rank),
                           prng_instances=16384)
    L = Q.Lattice(cfg)
    L.seed()
    L.init()
    L.sweep(2)                                  # leave the cold start before timing
    if args.shapes:
        tune = None
        L.set_shapes(*(int(x) for x in args.shapes.split(",")))
    else:
        tune = L.tune(reps=8)                   # launch shapes for this lattice (field restored)
    stream = torch.cuda.ExternalStream(L.stream())
    V = args.size ** 4
    updates_per_step = 4 * V * (1 + N_OR)

    for _ in range(args.warmup):
        L.sweep(1)
    L.sync()
    clocks = ClockSampler(local)
    clocks.start()
    RP.barrier(dist)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    L.sweep(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = RP.max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    RP.barrier(dist)
    clk = clocks.stop()
    value = RP.whole_job_rate(world, updates_per_step * args.steps, ms / 1e3)

    # dominant kernel: heatbath / overrelaxation phase launches back to back
    # between two events (as inside the sweep graph, so no per-launch gap is
    # counted), cycling over the 8 phase classes; three such runs, the median
    def time_phases(kind, reps=32):
        runs = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for i in range(reps):
                L.phase(i % 2, (i // 2) % 4, kind)
            e1.record(stream)
            torch.cuda.synchronize()
            runs.append(e0.elapsed_time(e1) / reps)
        return statistics.median(runs)

    ms_hb_alone = time_phases(Q.HEATBATH)
    ms_or_alone = time_phases(Q.OVERRELAX)
    # each kernel as it runs in the timed sweeps: its share of the sweep
    # graph (event nodes before and after every phase launch and around the
    # graph; 20 sweeps of the chain per call, median of 3 calls) times the
    # timed region's ms per sweep -- the share, not the absolute, carries
    # over, because the SM clock under load differs between the timed
    # region and any later measurement and both kernels follow it.  The
    # RANLUX mode keeps the back-to-back launches.
    ms_hb, ms_or, graph_times, how = ms_hb_alone, ms_or_alone, None, (
        "CUDA events on the library stream around 32 back-to-back phase launches per kind (median of 3), right "
        "after the timed region, same lattice and shapes")
    if prng == Q.PRNG_PHILOX:
        inside = [L.sweep_phase_times(20) for _ in range(3)]
        g_hb, g_or, g_sw = (statistics.median(t[i] for t in inside) for i in range(3))
        step_ms = ms / args.steps
        ms_hb, ms_or = g_hb / g_sw * step_ms, g_or / g_sw * step_ms
        graph_times = {"ms_per_launch_hb": g_hb, "ms_per_launch_or": g_or, "ms_per_sweep": g_sw,
                       "share_hb": 8 * g_hb / g_sw, "share_or": 8 * N_OR * g_or / g_sw}
        how = ("share of the sweep graph x the timed region's ms per sweep: qg_sweep_phase_times (CUDA event nodes "
               "before and after every phase launch and around the graph, 20 sweeps per call, median of 3 calls, "
               "right after the timed region, same lattice and shapes) gives each kernel's in-graph duration "
               "over the graph's ms per sweep (graph_times)")
    share_hb, share_or = 8 * ms_hb, 8 * N_OR * ms_or
    dom, dom_ms = ("heatbath", ms_hb) if share_hb >= share_or else ("overrelaxation", ms_or)
    alg_bytes = 4.5 * V * LINK_BYTES                # per phase launch (compulsory traffic)
    peak, peak_kind = peaks()
    achieved = alg_bytes / (dom_ms / 1e3) / 1e9
    traffic = None
    tr = profile_traffic()
    if tr and dom in tr:
        traffic = tr[dom]["dram_bytes_per_site"] * V / 2

    # end to end through the C-ABI: per step the run parameters go host ->
    # device from pinned staging (qg_set_params), one sweep, and the step's
    # plaquette sums -- FP32 products, FP64 sums (QG_MEAS_PLAQUETTE_F32) --
    # come back to pinned host memory (qg_measure_enqueue);
    # the host reads every step's values (qg_measure_fetch) -- one step
    # behind, so the device does not idle between steps -- and the timed
    # region ends when the last step's values are on the host
    e2e_steps = max(3, args.steps // 2)
    L.sync()
    RP.barrier(dist)
    e2e_plaq = []
    t0 = time.perf_counter()
    pending = None
    for _ in range(e2e_steps):
        L.set_params(BETA)
        L.sweep(1)
        tk = L.measure_enqueue(Q.MEAS_PLAQUETTE_F32)
        if pending is not None:
            e2e_plaq.append(L.measure_fetch(pending))
        pending = tk
    e2e_plaq.append(L.measure_fetch(pending))
    t1 = time.perf_counter()
    assert len(e2e_plaq) == e2e_steps
    e2e_s = RP.max_over_ranks(t1 - t0, dist, "cuda")
    e2e = RP.whole_job_rate(world, updates_per_step * e2e_steps, e2e_s)

    plq = L.plaquette()
    # the e2e readback's plaquette against the FP64-product one, same field,
    # and the device time of each (20 queued measurements between two
    # events, kernels and result copy; median of 3)
    p64, p32 = L.plaquette_sums(), L.plaquette_sums_f32()
    plq_dev = max(abs(a - b) for a, b in zip(p32, p64)) / (3 * 3 * V)

    def time_measure(kind, reps=20):
        runs = []
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            tks = [L.measure_enqueue(kind) for _ in range(reps)]
            e1.record(stream)
            torch.cuda.synchronize()
            for t in tks:
                L.measure_fetch(t)
            runs.append(e0.elapsed_time(e1) / reps)
        return statistics.median(runs)

    plq_ms = {"fp32_products": time_measure(Q.MEAS_PLAQUETTE_F32), "fp64_products": time_measure(Q.MEAS_PLAQUETTE)}
    L_shapes = L.shapes()
    first = 2 + args.warmup
    reunits = sum(1 for n in range(first + 1, first + args.steps + 1) if n % REUNIT_EVERY == 0)
    launches = args.steps * (8 + 8 * N_OR + (1 if prng == Q.PRNG_PHILOX else 0)) + reunits
    if prng == Q.PRNG_RANLUX:
        launches += 8 * args.steps
    L.close()
    RP.finish(dist)
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (cold start, %d untimed sweeps)" % (2 + args.warmup),
        "config": {"workload": "SU(3) %d^4 beta=%.1f, FP32 12-real links, 1 HB + %d OR per sweep, FP64 reunit every %d"
                               % (args.size, BETA, N_OR, REUNIT_EVERY),
                   "global_batch": world, "lattice": [args.size] * 4, "prng": args.prng,
                   "parallelism": "replicas x%d" % world,
                   "l2": ("field %.0f MB > 126 MB L2, no flush" if 4 * V * LINK_BYTES > 126e6 else
                          "field %.0f MB fits the 126 MB L2 (small-lattice run)") % (4 * V * LINK_BYTES / 1e6)},
        "roofline": {"bound": "hbm", "kernel": dom + " phase", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": alg_bytes, "ms_per_launch": dom_ms,
                     "ms_per_launch_hb": ms_hb, "ms_per_launch_or": ms_or,
                     "ms_per_launch_how": how,
                     # the same kernels launched one by one, back to back (the launch gaps the graph hides)
                     "ms_per_launch_hb_standalone": ms_hb_alone, "ms_per_launch_or_standalone": ms_or_alone,
                     "graph_times": graph_times,
                     # the literature's per-update count with no reuse between sites (19 link reads + 1
                     # write); above the HBM peak because neighbouring sites share their links in L2
                     "naive_bytes_per_update": 20 * LINK_BYTES,
                     "naive_gbs": 20 * LINK_BYTES * (V / 2) / (dom_ms * 1e-3) / 1e9},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 32, "d2h_bytes_per_step": 16,
                "what": "qg_set_params + qg_sweep + the step's plaquette sums read back (qg_measure_enqueue / "
                        "_fetch, one step behind), host wall clock",
                "plaquette": "FP32 products, FP64 sums (QG_MEAS_PLAQUETTE_F32)",
                "plaquette_dev_vs_fp64_products": plq_dev,
                "plaquette_ms": plq_ms},
        "gpu_launches": launches,
        "tuning_ms_per_launch": tune,
        "shapes": list(L_shapes),
        "clocks": clk,
        "plaquette": plq[2],
    }
    if not args.no_cpu_baseline and world == 1:
        # side measurements after the timed region: a failure in one of them
        # is reported in its own key and does not cost the bench line
        for key, leg in (("cpu_baseline", lambda: cpu_baseline_line(args.size)),
                         ("like_for_like", lambda: like_for_like(Q, torch, args.size))):
            try:
                line[key] = leg()
            except (RuntimeError, OSError, ValueError, Q.QGError) as e:
                line[key] = {"unavailable": "%s: %s" % (type(e).__name__, e)}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
