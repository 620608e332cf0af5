"""bench.py's output line: the keys the benchmark contract names, on a small
lattice -- the reference arm on the host (CPU), our arm on the GPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + list(args), cwd=ROOT,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_reference_arm_line():
    d = _bench("--impl", "reference", "--size", "8", "--steps", "2", "--warmup", "1")
    assert d["impl"] == "reference"
    if "unavailable" in d:
        pytest.skip(d["unavailable"])
    assert d["value"] > 0 and d["unit"] == "link_updates/s" and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["lattice"] == [8, 8, 8, 8]
    assert d["steps"] == 2 and d["steps_requested"] == 2



def test_reference_arm_reports_a_failing_reference_process(tmp_path, monkeypatch, capsys):
    """a reference CPU process that exits with an error gives the arm's
    "unavailable" line and status 0, not a traceback"""
    sys.path.insert(0, ROOT)
    import bench
    fake = tmp_path / "ref_cpurun"
    fake.write_text("#!/bin/sh\nexit 3\n")
    fake.chmod(0o755)
    monkeypatch.setattr(bench, "ref_binary", lambda: str(fake))
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--size", "4", "--steps", "2",
                                      "--warmup", "1"])
    args = bench.parse()
    assert bench.run_reference_arm(args) == 0
    d = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert d["impl"] == "reference" and "reference CPU path failed" in d["unavailable"]

def test_reference_arm_caps_its_timed_steps():
    """one reference step is a whole heatbath phase per process (about a
    second at 32^4), so a long --steps request is cut to the cap"""
    sys.path.insert(0, ROOT)
    import bench
    d = _bench("--impl", "reference", "--size", "4", "--steps", str(bench.REF_MAX_STEPS + 5), "--warmup", "1")
    if "unavailable" in d:
        pytest.skip(d["unavailable"])
    assert d["steps"] == bench.REF_MAX_STEPS and d["steps_requested"] == bench.REF_MAX_STEPS + 5
    assert d["value"] > 0


@pytest.mark.gpu
def test_our_arm_line():
    d = _bench("--size", "16", "--steps", "5", "--warmup", "3", "--no-cpu-baseline")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "e2e", "gpu_launches", "clocks"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 5 and d["warmup"] == 3 and d["value"] > 0
    assert d["value"] == pytest.approx(4 * 16 ** 4 * 5 / (d["ms_per_step"] * 1e-3), rel=1e-9)
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["achieved"] > 0 and r["peak"] > 0
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    # kernel times as they run in the timed sweeps: share of the sweep graph x timed ms per step
    g = r["graph_times"]
    for kind in ("hb", "or"):
        assert r["ms_per_launch_" + kind] == pytest.approx(g["ms_per_launch_" + kind] / g["ms_per_sweep"]
                                                           * d["ms_per_step"])
        assert r["ms_per_launch_%s_standalone" % kind] > 0
    assert g["share_hb"] == pytest.approx(8 * g["ms_per_launch_hb"] / g["ms_per_sweep"])
    assert 0 < g["share_hb"] + g["share_or"] < 1
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    assert 0 <= e["plaquette_dev_vs_fp64_products"] <= 1e-6
    assert set(e["plaquette_ms"]) == {"fp32_products", "fp64_products"}
    assert d["gpu_launches"] == 5 * (8 + 8 * 4 + 1) + sum(1 for n in range(6, 11) if n % 10 == 0)
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(d["clocks"])
    assert "workload" in d["config"] and "fits the 126 MB L2" in d["config"]["l2"]


def test_like_for_like_row_conversion_equals_the_oracles():
    """bench.py hands the reference CPU path its thermalised start in the
    reference's stored-row format; the conversion equals the oracle's"""
    import numpy as np

    import _oracle as O
    import bench
    c = O.make_cfg(group=3, dims=(4, 4, 4, 4), precision=1, beta=6.0, row_align=64)
    t = np.random.default_rng(3).standard_normal(12 * c.rowsize * 4)
    assert np.array_equal(bench.table_rows_fp64(t, 4, c.rowsize), O.table_to_rows(c, t))
