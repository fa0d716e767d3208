"""The bench's reference arm on the CPU: `bench.py --impl reference` prints one JSON line
with the keys the measurement contract names (metric, value, unit, steps, timing, config,
cpu_baseline, a zero-copy e2e block), and under a multi-rank launch only rank 0 prints."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--n-reads", "20000", "--steps", "1",
           "--warmup", "3"]
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_the_contract_line():
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    if "unavailable" in d:
        pytest.skip(d["unavailable"])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["metric"] == "reads/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 3
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_do_no_work():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_loads_no_mapping_code():
    # the reference arm's inputs come from the generator library alone: the process never
    # maps libdnaln_b200.so, so what it times is the reference's code only
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--n-reads', '5000', '--steps', '1', "
            "'--warmup', '0']; runpy.run_path('bench.py', run_name='__main__'); "
            "m = open('/proc/self/maps').read(); "
            "print('MAPS', 'libdnaln_b200.so' in m, 'libdnaln_synth.so' in m, 'libdnaln_ref.so' in m)")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("MAPS")][0]
    product, generator, reference = line.split()[1:]
    assert product == "False" and generator == "True"
