"""bench.py's reference arm (`--impl reference`): the reference's own CPU
code (oracle/_ref, the unmodified reference compiled here) timed on the host
cores for each workload, printing one JSON line with the keys of the bench
contract: the same metric and unit as the GPU arm, `impl` "reference", a
`cpu_baseline` describing the run and an `e2e` equal to the value with no
host-device copies.  Short runs (one timed step) on the CPU."""
import json
import os
import subprocess
import sys

import pytest

from oracle import ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) absent")

KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


def reference_line(*extra):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", *extra], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    return json.loads(lines[0])


@needs_ref
@pytest.mark.parametrize("workload", ["multichannel", "vegas", "batched", "large"])
def test_reference_arm_prints_the_contract_line(workload):
    d = reference_line(*(() if workload == "multichannel" else ("--workload", workload)))
    assert d["impl"] == "reference"
    for k in KEYS:
        assert k in d, k
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 0
    assert d["higher_is_better"] is True and d["dtype"] == "f64"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert isinstance(d["config"], dict) and d["config"].get("workload")
