"""bench.py's --gpus contract on the CPU: a run never reports fewer GPUs than it was asked for.
With no launcher it spawns its ranks itself (torch.distributed.run); a launcher whose world
size differs from --gpus, or fewer visible CUDA devices than --gpus, ends the run with an
error before any work."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(args, env_extra=None):
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                          env=env, timeout=120)


def test_world_size_mismatch_is_an_error():
    r = _bench(["--gpus", "2"], {"WORLD_SIZE": "1", "RANK": "0", "LOCAL_RANK": "0"})
    assert r.returncode != 0
    assert "--gpus 2 but the launcher started 1 ranks" in r.stderr


def test_more_gpus_than_devices_is_an_error():
    import torch
    have = torch.cuda.device_count()
    n = max(2, have + 1)
    r = _bench(["--gpus", str(n)])
    assert r.returncode != 0
    assert f"--gpus {n} but {have} CUDA devices are visible" in r.stderr


def test_zero_gpus_is_an_error():
    r = _bench(["--gpus", "0"])
    assert r.returncode != 0 and "--gpus must be >= 1" in r.stderr
