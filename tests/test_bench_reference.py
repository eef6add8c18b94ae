"""The reference arm of bench.py on the host: `--impl reference` times the
CPU FFT (the FP64 oracle, the reference's own HIP code cannot be built) on
a bounded sample and prints one JSON line with the same metric as the GPU
arm, `impl: reference`, a `cpu_baseline` describing the run and an `e2e`
with no host-device bytes; under torchrun only rank 0 runs and prints.
Sized to the small 1D 4096 x 256 workload (a few seconds)."""
import json
import os
import subprocess
import sys

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")


def _bench(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--config", "c1",
                           "--steps", "1", "--warmup", "3"], cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=300)


def test_reference_arm_json_line():
    r = _bench({})
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    with open(os.path.join(ROOT, "BASELINE.json")) as f:
        assert line["metric"] == json.load(f)["metric"]
    assert line["impl"] == "reference"
    assert line["unit"] == "GFLOP/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["n_gpus"] == 1 and line["steps"] == 1 and line["warmup"] >= 3
    assert line["config"]["dims"] == [4096] and line["config"]["batch"] == 256
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == line["value"] and cb["unit"] == line["unit"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    r = _bench({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
