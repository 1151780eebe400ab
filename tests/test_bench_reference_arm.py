"""bench.py's reference arm runs on the host cores (no GPU): one JSON line with
the contract's keys on rank 0, nothing on the other ranks.  Warm-up steps are
at least 3 whatever is asked (the timing rule)."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line():
    (line,) = run({})
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["warmup"] == 3 and line["steps"] == 1 and line["dtype"] == "f64"
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["ne"] == 32768 and line["config"]["nm"] == 28


def test_reference_arm_other_ranks_print_nothing():
    assert run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []


def test_reference_arm_does_not_load_the_cuda_library():
    """The reference arm sets the workload up with the oracle alone: the
    product library is never mapped into its process."""
    code = (
        "import sys, types\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1']\n"
        "import bench\n"
        "bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('LOADED' if 'libspoc_gpu.so' in maps else 'NOT_LOADED')\n"
    )
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "NOT_LOADED"
