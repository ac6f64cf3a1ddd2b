"""bench.py's JSON line, checked on the arm that runs without a GPU: the
reference's own CPU path (`--impl reference`) on a 16^3 system.  The keys
and their meanings are those the GPU arm prints too."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_complete_json_line():
    """Also: the arm loads no CUDA code (the system comes from the host-only
    build of the generator)."""
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--n", "16", "--steps", "2",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "time_to_true_rel_residual_1e-8" and d["unit"] == "s"
    assert d["higher_is_better"] is False and d["value"] > 0
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (1, 2, 3)
    assert d["requested"] == {"steps": 2, "warmup": 3} and len(d["step_times_s"]) == 2
    # every timed step is a complete solve to the tolerance
    assert d["converged"] is True and d["true_rel_residual"] < 1e-8 * 1.5
    assert set(d["solution_digest"]) == {"norm2", "sum", "dot_pm1"}
    assert abs(d["ms_per_step"] - 1e3 * d["value"]) < 1e-9 * max(1.0, d["ms_per_step"])
    assert d["scaling"] in ("weak", "strong") and d["vs_baseline"] is None
    assert d["dtype"] == "f64" and "synthetic" in d["data"]
    assert d["config"]["workload"].startswith("diffusion3d_16^3") and d["config"]["rows"] == 16 ** 3
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == "s" and cb["kind"] in ("reference", "port")
    assert cb["cores"] >= 1 and cb["sample"] and cb["nproc"] >= 1 and "cpu_model" in cb
    assert "complete solve" in cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == "s"
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
