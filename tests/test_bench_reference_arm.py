"""The benchmark's reference arm (`bench.py --impl reference`) on the host cores: the
reference algorithm (the CPU restatement under oracle/, the reference's Metal path
being unable to run here) timed on the benchmark's own workload. It prints one JSON
line with the GPU arm's metric, unit and workload, `impl` "reference", a cpu_baseline
that describes the run and an end-to-end rate without device copies; under a
multi-rank launch only rank 0 works and prints."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(extra_env):
    env = dict(os.environ, **extra_env)
    return subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                           "--steps", "1", "--warmup", "3"],
                          capture_output=True, text=True, timeout=900, env=env, cwd=REPO)


def _lines(out):
    return [json.loads(line) for line in out.splitlines() if line.startswith("{")]


def test_reference_arm_prints_one_line_of_the_benchmark_metric():
    p = _run({})
    assert p.returncode == 0, p.stderr[-2000:]
    lines = _lines(p.stdout)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference"
    assert d["metric"].startswith("SGM Gpixel-disparities/s") and d["unit"] == "Gpd/s"
    assert d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["config"]["workload"].startswith("c2: 64 mixed pairs")
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert "strata" in cb["sample"]


def test_reference_arm_other_ranks_exit_without_work():
    p = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert _lines(p.stdout) == []
