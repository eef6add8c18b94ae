"""The reference arm of bench.py on the host: `--impl reference` times the
CPU FFT (scipy.fft, standing in for the FFTW the reference's accuracy
harness calls; the reference's own HIP code cannot be built) over whole
steps of the workload and prints one JSON line with the same metric as the
GPU arm, `impl: reference`, a `cpu_baseline` describing the run and an
`e2e` with no host-device bytes; under torchrun only rank 0 runs and
prints.  Sized to the small 1D 4096 x 256 workload (a few seconds).  Also
the launch checks of the GPU arm that need no GPU: --gpus against the
launcher's world size, and the command that relaunches the script with one
rank per GPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")


def _bench(env_extra, args=("--impl", "reference", "--config", "c1", "--steps", "1",
                             "--warmup", "3")):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", *args], cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=300)


def test_reference_arm_json_line():
    r = _bench({})
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    # the GPU arm's metric (bench.METRIC), read from the script's source so
    # that nothing here imports torch
    with open(os.path.join(ROOT, "bench.py")) as f:
        src = f.read()
    metric = src.split('METRIC = "', 1)[1].split('"', 1)[0]
    assert line["metric"] == metric
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
    # whole steps: the measured time per step times the step's flops is the value
    flops = 5.0 * 4096 * 12 * 256
    assert abs(flops / (line["ms_per_step"] * 1e-3) / 1e9 - line["value"]) < 0.01 * line["value"]
    assert "whole workload" in cb["sample"]


def test_reference_arm_other_ranks_exit_quietly():
    r = _bench({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_gpus_must_match_the_launchers_world_size():
    """Under a launcher, --gpus N with WORLD_SIZE != N is an error (exit 2)
    before any device is touched."""
    r = _bench({"RANK": "0", "WORLD_SIZE": "2", "LOCAL_RANK": "0"},
               ("--gpus", "4", "--steps", "1", "--warmup", "3"))
    assert r.returncode == 2, (r.returncode, r.stderr)
    assert "WORLD_SIZE=2" in r.stderr


def test_gpus_relaunch_command():
    """Without a launcher, --gpus N > 1 reruns the script under
    torch.distributed.run with N ranks on this node (127.0.0.1)."""
    sys.path.insert(0, ROOT)
    import bench
    cmd = bench.relaunch_cmd(["--gpus", "8", "--steps", "5"], 8, 29511)
    assert cmd[1:3] == ["-m", "torch.distributed.run"]
    assert "--nproc-per-node=8" in cmd and "--nnodes=1" in cmd
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[cmd.index("--master-port") + 1] == "29511"
    assert cmd[-4:] == ["--gpus", "8", "--steps", "5"]
    assert cmd[-5].endswith("bench.py")
