"""The bench's reference arm (the CPU implementation of the same SCF, timed on
the host) keeps the line contract: one JSON line with impl, metric, value,
unit, cpu_baseline and an e2e object with zero host-device bytes.  A small
case (16 waters, 8 alkanes) keeps it to seconds."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    env = dict(os.environ, OPENBLAS_NUM_THREADS="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1", "--nwater", "16", "--batch", "8"],
                         capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "scf_single_points_per_s" and d["unit"] == "SCF/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "SCF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["batched"]["value"] > 0
    # one complete oracle SCF in the GPU arm's mode, reported as equal slices
    assert d["scf"]["converged"] and d["scf"]["niter"] > 4
    assert abs(d["ms_per_step"] * d["steps"] / 1e3 - d["scf_wall_s"]) < 1e-6
    assert d["plain_mode"]["niter"] > 4
    assert d["config"]["mode"] == "fast" and d["config"]["finish_dp"] == 1e-7
