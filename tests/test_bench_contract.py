"""bench.py's reference arm (--impl reference): the reference's CPU implementation
of the path timed on the host cores.  It runs without a GPU, so its JSON line is
checked here: one line from rank 0 with the metric, unit and direction of the
GPU arm, a cpu_baseline block describing the sample, an e2e block with no
host-device traffic, and every timed step a full solve of the GPU arm's
workload (here at n = 2048 to keep the test short); other ranks print nothing and exit 0."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _run(env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                           "--n", "2048"],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    import bench

    r = _run({})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"] and cb["kind"] in ("port", "reference")
    assert cb["cores"] >= 1 and "dpotrf" in cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    # the GPU arm's workload string: the same configuration, timed at full size
    assert d["config"]["workload"] == "pposv d uplo=L n=2048 nrhs=8 A=U diag(s) U^T kappa=1e+06"
    assert "1 full solves at n=2048" in cb["sample"]


def test_reference_arm_other_ranks_are_silent():
    r = _run({"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_clock_summary_decodes_reasons_and_median():
    """The clock record of the timed region: NVML reason bits map to the names the
    timing rules use (hw_slowdown 0x8, hw_thermal_slowdown 0x40, sw_thermal_slowdown
    0x20, sw_power_cap 0x4), and the SM clock reported is the median of the samples."""
    import pynvml

    import bench

    assert dict(bench.ClockSampler.REASON_BITS) == {
        "hw_slowdown": pynvml.nvmlClocksThrottleReasonHwSlowdown,
        "hw_thermal_slowdown": pynvml.nvmlClocksThrottleReasonHwThermalSlowdown,
        "sw_thermal_slowdown": pynvml.nvmlClocksThrottleReasonSwThermalSlowdown,
        "sw_power_cap": pynvml.nvmlClocksThrottleReasonSwPowerCap,
    }
    c = bench.ClockSampler(0)
    c.samples = [(1965.0, 0x0), (1890.0, 0x4), (1920.0, 0x4 | 0x1)]
    c.max_mhz = 1965.0
    s = c.summary()
    assert s["sm_mhz"] == 1920.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"] and s["source"] == "nvml"
    c.samples = [(1400.0, 0x40 | 0x8)]
    assert bench.ClockSampler.summary(c)["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]
