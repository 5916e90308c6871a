"""The reference arm of bench.py on the host: its JSON line keeps the contract.

`bench.py --impl reference` times the FP64 OpenMP oracle (the restatement of
ph_scattering.cpp's builder) on a bounded q2 sample of the 20^3 headline
workload.  Its line must carry the GPU arm's `config`, `metric`, `unit` and
`higher_is_better`, say that its step time is projected from the sample, and
describe the sample in `cpu_baseline`.  No GPU is needed."""
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def line():
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4"))
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--cpu-seconds", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def test_reference_line_keeps_the_contract(line):
    assert line["impl"] == "reference"
    assert line["metric"] == "3ph triplets/s @20^3 mesh"
    assert line["unit"] == "triplets/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 0
    assert line["projected_from_sample"] is True
    nq = 20 ** 3
    assert abs(line["ms_per_step"] - 1000.0 * nq * nq / line["value"]) <= 1e-6 * line["ms_per_step"]
    assert line["e2e"] == {"value": line["value"], "unit": "triplets/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == line["value"] and cb["cores"] >= 1
    assert "q2 points" in cb["sample"]


def test_reference_line_has_the_gpu_arms_config(line):
    sys.path.insert(0, ROOT)
    import bench
    assert line["config"] == bench.headline_config(20, 43, "split_fp16", 1)
