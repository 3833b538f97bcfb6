"""The benchmark's reference arm runs on the CPU alone: its JSON line keeps
the result contract (impl, metric, value, unit, cpu_baseline, e2e) for the
default workload and for the batch and elasticity samples.  It times the
compiled reference (oracle/_ref) and skips where that was not built."""
import json
import os
import subprocess
import sys

import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _line(*extra):
    if not os.path.exists(O.REF_HARNESS):
        pytest.skip("reference harness not built (make -C oracle ref)")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1", *extra],
                         capture_output=True, text=True, timeout=900, check=True).stdout
    lines = [ln for ln in out.strip().splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out
    return json.loads(lines[0])


@pytest.mark.parametrize("workload", ["grid3d", "batch", "elasticity"])
def test_reference_arm_line(workload):
    d = _line("--workload", workload)
    assert d["impl"] == "reference" and d["unit"] == "GFLOP/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 1
    base = d["cpu_baseline"]
    assert base["kind"] == "reference" and base["cores"] >= 1 and base["sample"]
    assert base["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_sub_workloads_record_lines_failures_and_time_limits(tmp_path):
    """The default single-GPU run carries its adjoint and elasticity lines
    under "workloads" by running each mode as a child process; a child's
    last JSON line is kept, and a child that fails or overruns its time limit
    leaves an error entry instead of stopping the bench."""
    sys.path.insert(0, ROOT)
    import bench

    script = tmp_path / "child.py"
    script.write_text(
        "import json, sys, time\n"
        "mode = sys.argv[1]\n"
        "if mode == 'ok':\n"
        "    print('log line'); print(json.dumps({'metric': 'm', 'value': 1.5}))\n"
        "elif mode == 'fail':\n"
        "    sys.stderr.write('boom'); sys.exit(3)\n"
        "else:\n"
        "    time.sleep(30)\n")
    out = bench.run_sub_workloads(
        workloads=(("a", ["ok"]), ("b", ["fail"]), ("c", ["slow"])), timeout_s=2.0,
        script=str(script))
    assert out["a"]["value"] == 1.5 and out["a"]["wall_s"] >= 0
    assert out["b"]["error"].startswith("exit 3") and "boom" in out["b"]["error"]
    assert "timed out" in out["c"]["error"] and out["c"]["wall_s"] < 20
    assert [w for w, _ in bench.SUB_WORKLOADS] == ["adjoint", "elasticity"]
