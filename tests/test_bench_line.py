"""CPU: bench.py's output contract.

* The printed result line stays small (the driver keeps only the tail of
  stdout): a result with every key the B200 arm fills, at realistic sizes,
  must print well under 4 KB, and the per-class table must not be part of it.
* The reference arm loads no part of the B200 library: it builds its
  workload from simint_b200/workloads.py by file path and runs the
  reference's generated library (oracle/_ref).
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def fake_result():
    cls = {"am": "fdfp", "ms": 8.2234567, "tflops": 0.971234567}
    return {
        "metric": bench.METRIC, "value": 5.1612345e8, "unit": "primitive quartets/s",
        "n_gpus": 1, "steps": 20, "warmup": 5, "ms_per_step": 80.0512345, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32 (FP32 VRR behind the per-integral error gate)",
        "data": "synthetic (seeded cfg2 shells, PCG64 seed 2024)",
        "config": dict(bench.workload_config(bench.parse([])), quartets_per_step=1220482,
                       primq_per_step=41345678, full_sweep_quartets=1912345678, gate=1e-10,
                       l2="256 MB flush before every timed step", setup_s=12.3, autotune_s=45.6),
        "fp64": {"value": 5.0612345e8, "ms_per_step": 81.6712345},
        "vs_reference_values": {"fp64": {"max_abs": 3.1e-14, "max_rel": 2.2e-12, "quartets": 1220000,
                                         "bar_failures": 0},
                                "mixed": {"max_abs": 8.1e-11, "max_rel": 3.3e-6, "quartets": 1220000,
                                          "bar_failures": 12345},
                                "reference": "gamess_l3", "bar": "abs <= 1e-13 or rel <= 1e-11 (fp64); "
                                "mixed: max abs <= gate", "gate": 1e-10},
        "roofline": {"bound": "fp64", "kernel": "class fdfp", "achieved": 0.97123, "peak": 34.1234,
                     "unit": "TFLOP/s", "frac": 0.02845, "traffic": 123456789.0,
                     "peak_source": "measured FP64 FMA-chain probe, of measured"},
        "top_classes": [cls, cls, cls],
        "cpu_baseline": {"value": 2.5e7, "unit": "primitive quartets/s", "cores": 16, "kind": "reference",
                         "sample": "the same 182 sampled rows (4.58e+07 primitive quartets, 1.80 s per pass, "
                                   "3 passes), reference gamess_l3 build"},
        "e2e": {"value": 8.6e7, "unit": "primitive quartets/s", "h2d_bytes_per_step": 1400000000,
                "d2h_bytes_per_step": 1400000000, "calls_per_step": 55, "primq_per_step": 22800000},
        "gpu_launches": 2200,
        "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 30},
    }


def test_line_is_compact_and_parses():
    line = bench.compact(fake_result())
    assert len(line) < 2500, len(line)
    d = json.loads(line)
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "roofline",
              "cpu_baseline", "e2e", "gpu_launches", "clocks"):
        assert k in d, k
    assert "per_class" not in d
    assert d["vs_baseline"] is None


def test_line_limit_enforced():
    r = fake_result()
    r["per_class"] = [{"am": "x" * 50, "v": float(k)} for k in range(200)]
    with pytest.raises(ValueError):
        bench.compact(r)


def test_reference_arm_loads_no_b200_code():
    """The reference arm's imports (oracle/reflib, oracle/refsweep and the
    workload module by path) leave simint_b200 unimported and
    libsimint_b200.so unloaded."""
    code = (
        "import sys, os; sys.path.insert(0, %r); import bench; "
        "reflib, refsweep, R = bench.load_reference(); "
        "sh = refsweep.workloads().config_shells('cfg2'); "
        "maps = open('/proc/self/maps').read(); "
        "print('simint_b200' in sys.modules, 'libsimint_b200' in maps, len(sh))" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["False", "False", "500"], r.stdout
