"""bench.py's reference arm on the CPU: one JSON line with the keys of the
benchmark contract, on the seeded population and on a population file; under
torchrun the ranks other than 0 exit without output."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                       capture_output=True, text=True, timeout=300, cwd=ROOT, env=e)
    assert r.returncode == 0, r.stdout + r.stderr
    return [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]


def check_line(d):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["warmup"] >= 3 and "workload" in d["config"]
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["cpu_baseline"]["cores"] >= 1 and d["cpu_baseline"]["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_line():
    (d,) = run_bench("--steps", "1", "--warmup", "3", "--n-objects", "3000", "--reference-budget", "1")
    check_line(d)
    assert d["config"]["n_objects"] == 3000 and d["data"].startswith("synthetic")


def test_reference_arm_on_population_file(tmp_path):
    from ladds_b200 import capi

    path = str(tmp_path / "pop.bin")
    capi.save_population(path, capi.generate_population(0, 9, 2500))
    (d,) = run_bench("--steps", "1", "--warmup", "3", "--population", path, "--reference-budget", "1")
    check_line(d)
    assert d["config"]["n_objects"] == 2500 and d["data"] == "population file"
    assert "pop.bin" in d["config"]["workload"]


def test_reference_arm_loads_no_gpu_code_and_prints_the_gpu_arms_config():
    """The reference arm maps none of the package's GPU libraries (its
    population comes from the host-only generator), and its config dict is the
    one the GPU arm prints (bench.bench_config)."""
    code = (
        "import json, runpy, sys, io, contextlib\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3', '--n-objects', '2000',"
        " '--reference-budget', '1']\n"
        "buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf):\n"
        f"    runpy.run_path({os.path.join(ROOT, 'bench.py')!r}, run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'line': buf.getvalue(), 'gpu_lib': 'libladds_gpu' in maps,"
        " 'peaks_lib': 'libladds_peaks' in maps}))\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stdout + r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert not out["gpu_lib"] and not out["peaks_lib"]
    d = json.loads(out["line"].strip().splitlines()[-1])
    sys.path.insert(0, ROOT)
    import bench

    class A:
        population = None
        n_objects = 2000

    assert d["config"] == bench.bench_config(A, 2000)


def test_reference_arm_other_ranks_are_silent():
    assert run_bench("--steps", "1", "--warmup", "3", env={"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"}) == []
