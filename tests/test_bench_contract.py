"""The bench's CPU-side contract: the reference arm's JSON line (the oracle on the host's cores, in the
product arm's metric and unit) and the parsing of the autotuner's report."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def test_reference_arm_prints_one_line_in_the_product_metric():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "small_map",
                        "--steps", "1", "--warmup", "1", "--cpu-seconds", "1"],
                       capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "Grays/s" and d["unit"] == "Grays/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1
    assert d["config"]["workload"] == "small_map"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "Grays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_autotuner_report_parses():
    import bench
    rep = ("direct: bvh 2, refill 0, near 1, order 0, register cap 4, fetch 1, warp walk 0, 4 blocks/SM "
           "(4.403520 ms on 65536 texels); gather: bvh 2, refill 0, near 1, order 0, register cap 3, fetch 1, "
           "3 blocks/SM (4.789856 ms on 65536 texels); ")
    t = bench.parse_tuning(rep)
    assert t["direct"]["register cap"] == 4 and t["direct"]["near"] == 1 and t["direct"]["warp walk"] == 0
    assert t["gather"]["register cap"] == 3 and t["gather"]["bvh"] == 2
