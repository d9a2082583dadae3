"""bench.py's reference arm on the CPU: one JSON line with the keys of the
bench contract, the reference's own OpenMP RSVD timed on a bounded sample;
ranks other than 0 print nothing; a workload whose reference kernel cannot
run here says so in an `unavailable` line."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args,
                         cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line(ref):      # ref: the compiled reference exists
    lines = _run(["--impl", "reference", "--steps", "1", "--warmup", "0"])
    assert len(lines) == 1
    d = lines[0]
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup",
                "ms_per_step", "higher_is_better", "scaling", "vs_baseline",
                "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["steps"] == 1 and d["warmup"] == 0 and d["higher_is_better"]
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"].startswith("spatial-2d-sqexp-N102400")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_print_nothing():
    assert _run(["--impl", "reference", "--steps", "1", "--warmup", "0"],
                {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []


def test_reference_arm_unavailable_kernel(ref):
    lines = _run(["--impl", "reference", "--workload", "c2-matern",
                  "--steps", "1", "--warmup", "0"])
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and lines[0]["unavailable"]
