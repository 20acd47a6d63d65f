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


class _FakeNvml:
    """The NVML calls the bench's in-region clock sampler makes, answering with
    a fixed SM clock and a reason mask that turns on sw_power_cap (0x4) after
    the third sample."""
    NVML_CLOCK_SM = 1

    def __init__(self, fail_init=False):
        self.fail_init, self.calls, self.shut = fail_init, 0, False

    def nvmlInit(self):
        if self.fail_init:
            raise RuntimeError("no driver")

    def nvmlDeviceGetHandleByIndex(self, i):
        return ("gpu", i)

    def nvmlDeviceGetHandleByPciBusId(self, bus):
        raise RuntimeError("not found")  # the sampler falls back to the index

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        self.calls += 1
        return 1950 if self.calls % 2 else 1965

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return 0x4 if self.calls > 3 else 0x1

    def nvmlShutdown(self):
        self.shut = True


def test_nvml_clock_sampler_summary():
    import time
    sys.path.insert(0, ROOT)
    import bench
    nv = _FakeNvml()
    c = bench.NvmlClocks("00000000:3B:00.0", 0, period=0.001, nvml=nv)
    c.start()
    time.sleep(0.05)
    c.stop()
    s = c.summary()
    assert nv.shut and s["samples"] >= 4 and s["sm_max_mhz"] == 1965.0
    assert 1950.0 <= s["sm_mhz"] <= 1965.0
    # 0x1 (idle) is not a reported reason; 0x4 is sw_power_cap
    assert s["reasons"] == ["sw_power_cap"] and s["source"].startswith("NVML")


def test_nvml_clock_sampler_without_nvml():
    sys.path.insert(0, ROOT)
    import bench
    c = bench.NvmlClocks("0", 0, nvml=_FakeNvml(fail_init=True))
    c.start()
    c.stop()
    assert c.summary() is None
