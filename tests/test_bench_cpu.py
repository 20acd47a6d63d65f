"""bench.py's CPU arms: the reference arm (the CPU restatement of the
reference on the host cores) prints one JSON line with the contract's keys,
and under a multi-rank launch only rank 0 prints it."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                       timeout=300, env=e, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]


def test_reference_arm_line():
    (line,) = run(["--impl", "reference", "--steps", "1", "--warmup", "1", "--n", "24"])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 1
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["unit"] == line["unit"]
    assert line["config"]["workload"].startswith("tgv24:") and line["config"]["points"] == 25 ** 3


def test_reference_arm_other_ranks_print_nothing():
    assert run(["--impl", "reference", "--steps", "1", "--warmup", "0", "--n", "24"],
               env={"RANK": "1", "WORLD_SIZE": "2"}) == []
