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
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["metric"] == load_bench().METRIC and d["value"] > 0.0
    assert d["config"]["workload"] == "mac3d_reflection_maccormack_256"
    cpu = d["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["cores"] == 1 and cpu["value"] == d["value"] and cpu["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
