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


def test_panel_roofline_counts_every_eigensolve_order():
    """The dominant kernel's algorithmic bytes cover every eigensolve of the
    timed SCFs: the whole n for each full eigensolve, and the occupied and
    virtual orders for an exit diagonalisation solved as the two blocks."""
    from types import SimpleNamespace
    sys.path.insert(0, ROOT)
    import bench
    ctx = SimpleNamespace(norbs=3072, nclose=2048)
    results = [SimpleNamespace(n_full_diag=1, exit_split=True), SimpleNamespace(n_full_diag=2, exit_split=False)]
    sizes = bench.eigh_sizes(ctx, results)
    assert sizes == [3072, 2048, 1024, 3072, 3072]
    panels = sum((m - 2) // 32 + 1 for m in sizes)
    kst = {"tridiag_panel": {"launches": panels, "total_ms": 100.0}}
    r = bench.panel_roofline(ctx, kst, sizes)
    algo = sum(8.0 * (m - 1) * m * (2 * m - 1) / 6.0 for m in sizes)
    assert r["launches"] == r["launches_expected"] == panels
    assert abs(r["achieved"] - algo / 0.1 / 1e9) < 1e-6 * r["achieved"]
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert r["eigensolve_orders"] == [1024, 2048, 3072]
    # the DRAM traffic of a 3072 panel, scaled by algorithmic bytes
    one = bench.panel_roofline(ctx, {"tridiag_panel": {"launches": 96, "total_ms": 40.0}}, [3072])
    assert abs(one["traffic"] - bench.PANEL_DRAM_BYTES) < 1.0
