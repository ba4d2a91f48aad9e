"""Host-side parts of the benchmark's output contract, without a GPU: the
reference arm's JSON line (the reference's compiled CPU step) and the clock
sampler's reading of nvidia-smi lines."""
import importlib.util
import json
import os
import subprocess
import sys

import pytest

from oracle_lib import ref_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _FinishedProcess:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def test_clock_sampler_reads_median_and_reasons():
    bench = load_bench()
    s = bench.ClockSampler(0)
    s.proc = _FinishedProcess()
    s.lines = ["0, 1200, 1965, 300.0, 0x0, Not Active, Not Active, Not Active, Not Active",  # before timing
               "0, 1965, 1965, 950.5, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1905, 1965, 998.0, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1950, 1965, 990.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "garbage"]
    s.mark = 1
    info = s.stop()
    assert info == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}


def test_clock_sampler_without_samples_reports_none():
    bench = load_bench()
    s = bench.ClockSampler(0)
    assert s.stop() is None  # never started (no nvidia-smi)


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_reference_arm_prints_one_contract_line():
    # a small grid keeps the CPU suite fast; the driver runs it at 256^3
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--n", "32", "--reference-sweeps", "200"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["metric"] == load_bench().METRIC and d["value"] > 0.0
    assert d["config"]["workload"] == "mac3d_reflection_maccormack_32"
    cpu = d["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["cores"] == 1 and cpu["value"] == d["value"] and cpu["sample"]
    assert cpu["sweeps_charged"] == 200 and d["extrapolated"] is True
    # steps and ms_per_step describe the reference steps that actually ran
    assert d["steps"] == 2 and d["warmup"] == 1
    assert d["steps"] * d["ms_per_step"] <= d["wall_s"] * 1e3
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_charge_is_linear_in_sweeps_only():
    bench = load_bench()
    costs = {"n": 256, "fixed_s": 36.0, "per_sweep_s": 0.11,
             "timed_steps": [{"sweeps": 80, "seconds": 44.8}, {"sweeps": 16, "seconds": 37.76}]}
    line = bench.reference_line(costs, 5000.0, "test")
    assert line["value"] == pytest.approx(1.0 / (36.0 + 5000 * 0.11))
    assert line["measured_ms_per_step"] == pytest.approx(1e3 * (44.8 + 37.76) / 2)


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "vapor_b200", "tuning", "plain_sweeps.json")),
                    reason="plain-arm sweep table not recorded yet")
def test_plain_sweeps_window_matches_the_gpu_arm_steps():
    bench = load_bench()
    sweeps, table = bench.plain_sweeps_charged(5, 20)
    per_step = table["per_step"]
    window = [per_step[min(i, len(per_step) - 1)] for i in range(5, 25)]
    assert table["n"] == 256 and sweeps == pytest.approx(sum(window) / 20)
    assert all(isinstance(v, int) and v > 0 and v % 8 == 0 for v in per_step)
