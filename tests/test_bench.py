"""bench.py's output contract, checked on the CPU: the reference arm prints
one JSON line with the metric, unit, value, timing, config, cpu_baseline
and e2e keys the contract names (on the small workload, so it ends in
seconds); the closure workload's reference arm declares itself
unavailable; and the byte model behind `roofline` counts what the kernels
must move."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    d = run_bench("--impl", "reference", "--workload", "hydro-64x64x128", "--steps", "1", "--warmup", "3")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "cell-updates/s" and d["value"] > 0
    assert d["warmup"] >= 3 and d["config"]["workload"] == "hydro-64x64x128"
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


def test_closure_reference_arm_is_unavailable():
    d = run_bench("--impl", "reference", "--workload", "closure-64x128x256", "--steps", "1", "--warmup", "3")
    assert d["impl"] == "reference" and "unavailable" in d


def test_byte_model():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.step_alg_bytes(5) == 680 and bench.step_alg_bytes(8) == 1088
    # the radial sweep reads the five fields and the tendency and writes the tendency
    assert bench.kernel_alg_bytes("radial_terms", 5) == 8.0 * 15
    # the update kernel, averaged over the four stages
    assert bench.kernel_alg_bytes("rhot_update", 5) == 8.0 * (3 + 15 + 35 / 4.0)
    assert bench.kernel_alg_bytes("no_such_kernel", 5) is None
