"""bench.py's command-line contract on the CPU: the reference arm (`--impl reference`) runs the
reference's own CPU build of the force evaluation (or the oracle port where that build is
absent) on the same workload definition as the GPU arm and prints one JSON line with the keys
the bench contract names; under torchrun only rank 0 prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, env=None):
    e = dict(os.environ, OMP_NUM_THREADS="2")
    if env:
        e.update(env)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                       timeout=600, env=e, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]


def test_reference_arm_prints_the_contract_line():
    lines = _run(["--impl", "reference", "--n", "8192", "--steps", "2", "--warmup", "1"])
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "dtype", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["unit"] == "particle-steps/s" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["config"]["n"] == 8192 and d["config"]["p"] == 12
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["value"] == d["value"]
    # a workload other than the headline's is named by what it is
    assert "N=4M" not in d["metric"] and "N8192" in d["metric"]


def test_reference_arm_other_ranks_print_nothing():
    assert _run(["--impl", "reference", "--n", "4096", "--steps", "1", "--warmup", "1"],
                env={"RANK": "1", "WORLD_SIZE": "2"}) == []
