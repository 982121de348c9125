"""The bench's reference arm (CPU): it times the oracle port of the reference's kernels on the host
cores, prints one JSON line with the contract's keys, and maps no library of the product (its
scenes come from the oracle library's own copy of the generators)."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

SNIPPET = r"""
import json, sys, types
sys.argv = ["bench.py", "--impl", "reference", "--config", "cornell", "--steps", "1", "--warmup", "0"]
sys.path.insert(0, ".")
import bench
a = types.SimpleNamespace(steps=1, warmup=0, gpus=1, config="cornell")
line = bench.run_reference(a, bench.CONFIGS["cornell"])
maps = open("/proc/self/maps").read()
print(json.dumps({"line": line, "libphx": "libphx.so" in maps, "liboracle": "liboracle.so" in maps}))
"""


def test_reference_arm_contract_and_no_product_library():
    r = subprocess.run([sys.executable, "-c", SNIPPET], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["liboracle"] and not out["libphx"], "the reference arm must map the oracle library only"
    line = out["line"]
    assert line["impl"] == "reference" and line["metric"] == "Mphotons/s" and line["unit"] == "Mphotons/s"
    assert line["value"] > 0 and line["higher_is_better"] is True and line["n_gpus"] == 1
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["value"] == line["value"] and cpu["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"] == "cornell"
