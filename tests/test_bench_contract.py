"""bench.py's one JSON line, from both arms, on the small configuration (c1):
the keys and value kinds the benchmark contract names.  The reference arm runs
the reference's own CPU code on the host cores (no GPU); ours needs a B200."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
COMMON = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
          "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "e2e",
          "cpu_baseline"}


def _line(args, timeout):
    out = subprocess.run([sys.executable, "bench.py", *args], cwd=ROOT, capture_output=True,
                         text=True, timeout=timeout)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-3000:]
    return json.loads(lines[0])


def test_reference_arm_line():
    d = _line(["--impl", "reference", "--workload", "c1", "--steps", "1", "--warmup", "0"], 600)
    assert COMMON <= d.keys()
    assert d["impl"] == "reference" and d["unit"] == "vis/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["n_gpus"] == 1
    cpu = d["cpu_baseline"]
    assert cpu["kind"] in ("reference", "port") and cpu["cores"] >= 1 and cpu["sample"]
    assert cpu["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "vis/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    # the same workload keys as our arm's line; timed steps cover measured chunks
    assert {"workload", "rows", "visibilities", "grid", "w_planes", "kernel", "w_support",
            "l2", "parallelism", "time_fraction"} <= d["config"].keys()
    assert abs(d["ms_per_step"] * d["steps"] * 1e-3 * d["value"] -
               float(cpu["sample"].split("(")[1].split(" jobs")[0]) * d["config"]["visibilities"]
               ) / (d["config"]["visibilities"]) < 0.05


@pytest.mark.gpu
def test_our_arm_line():
    d = _line(["--workload", "c1", "--steps", "3", "--warmup", "3", "--no-served", "--no-batched"],
              900)
    assert (COMMON | {"roofline", "gpu_launches", "clocks"}) <= d.keys()
    assert d["unit"] == "vis/s" and d["value"] > 0 and d["warmup"] >= 3 and d["steps"] == 3
    assert d["dtype"] == "f64" and d["data"] == "synthetic" and d["scaling"] in ("weak", "strong")
    assert d["config"]["workload"] and d["gpu_launches"] > 0
    roof = d["roofline"]
    assert roof["bound"] in ("hbm", "tensor") and roof["unit"] in ("GB/s", "TFLOP/s")
    assert roof["achieved"] > 0 and roof["peak"] > 0
    assert abs(roof["frac"] - roof["achieved"] / roof["peak"]) < 1e-3
    e2e = d["e2e"]
    assert e2e["unit"] == "vis/s" and e2e["value"] > 0
    assert e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= d["clocks"].keys()
    forms = d["forms"]
    assert forms["mixed"]["rel_l2_vs_fp64"] < 1e-5
    # both forms against the CPU path's own image of the same job
    assert forms["vs_oracle"]["fp64"]["rel_l2"] < 1e-12
    assert forms["vs_oracle"]["mixed"]["rel_l2"] < 1e-5
    assert d["cpu_baseline"]["value"] > 0 and d["cpu_baseline"]["kind"] in ("reference", "port")
