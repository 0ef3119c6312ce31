#!/usr/bin/env python
"""Benchmark: PM7 1SCF on a seeded (H2O)_512 box (3072 basis functions, 2048
doubly occupied MOs) on one B200.

A step is one complete SCF -- the reference's iter from the standard diagonal
guess to self-consistence -- over the resident integrals (H, W computed once
on the GPU before timing; W is 151 MB, larger than L2, and L2 is flushed
between steps anyway).  The headline metric is SCF single points per second
(whole job); scf_wall_s is the time of one SCF.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--mode fast|plain]
                  [--precision split|fp64] [--impl mine|reference]

--mode fast   pseudo-diagonalisation once the reference's newdg switch is set
              (the path the reference comments out), full FP64 eigensolves
              otherwise -- the product path.
--mode plain  full FP64 eigensolve every iteration, like the fork's iter.
--precision split (default) density and Fmo GEMMs as three BF16 products on
              the tensor cores until max|dP| < 1e-4, FP64 after (convergence
              is only accepted in FP64); fp64: FP64 throughout.  The line
              states |dHf| of the timed SCF against the FP64 SCF and the time
              of the plain FP64 path (full eigensolve every iteration, FP64
              GEMMs) on the same box.
--impl reference
              times the CPU implementation of the same SCF (the oracle: C
              Fock build and rotation sweep, LAPACK dsyevd and BLAS through
              numpy) on the host cores: one complete SCF in the same mode
              (pseudo-diagonalisation, Pulay, finish to max|dP| <= 1e-7, all
              FP64), reported as --steps slices of that one timed SCF, plus a
              complete plain-mode SCF beside it; N > 1: rank 0 only.
--converger pulay (default in fast mode) Pulay's DIIS once newdg is set,
              like the PULAY keyword; cnvg: the default extrapolation.
--guess learned (default): each step starts from the atom-pair network
              trained on liquid-density boxes (prediction and one McWeeny step
              on the device, inside the timed region), entered like an OLDENS
              density; standard: the reference's diagonal guess.  The line
              reports under "learned_guess" the fast path from the other guess
              and a sample of the held-out (H2O)_n lattice-cluster evaluation
              (n = 32..128, plain FP64 path, standard vs learned guess).
--shift N     the reference's SHIFT=N keyword for the timed SCF (default 0 in
              fast mode: no level shift, newdg from the first small density
              change, SCF/iter.F90:131-136; "default" keeps iter's -80).  The
              plain FP64 reference point always runs iter's default keywords.
--mozyme N    also time the MOZYME SCF of a seeded (H2O)_N box (default 4096:
              12 288 atoms, 24 576 basis functions, CUTOFF=9): pair-block
              layout and integrals on the GPU, the water starting LMOs, the
              SCF loop behind mb_mz_scf_run to convergence; reported under
              "mozyme".  0 skips it.
--batch N     also measure the batched workload (default 4096 seeded linear
              alkanes C3-C20, one persistent launch, a CTA per molecule SCF):
              batched SCFs/s on device-resident integrals, the same through
              the C ABI from host coordinates (integrals included), the plain
              FP64 GPU path (one molecule at a time) and the CPU oracle on
              samples; reported under "batched".  0 skips it.
Multi-GPU: replicas only (independent SCFs per rank, no data-path
collective); the batched workload gives each rank its share of a list of
--batch x N alkanes (mopac_gpu_b200.replicas.shard), times are max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "(H2O)512 water box, PM7 1SCF, RHF closed shell, 1536 atoms, 3072 basis functions, 2048 occupied"
METRIC = "scf_single_points_per_s"
BATCH_WORKLOAD = ("linear alkanes C3H8..C20H42, seeded random staggered conformers (no syn-pentane pairs), "
                  "PM7 1SCF each, RHF closed shell, 11-62 atoms, 20-122 basis functions")
# FP64 finish of the split-precision SCF (mb_scf_opts.finish_dp), used by the
# oracle runs in the same mode
FINISH_DP = 1.0e-7


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--mode", choices=["fast", "plain"], default="fast")
    ap.add_argument("--precision", choices=["split", "fp64"], default="split")
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--nwater", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--guess", choices=["learned", "standard"], default="learned")
    ap.add_argument("--shift", default="0")
    ap.add_argument("--converger", choices=["pulay", "cnvg"], default="pulay")
    ap.add_argument("--guess-sample", type=int, default=40)
    ap.add_argument("--mozyme", type=int, default=4096)
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def oracle_system(nwater: int):
    """The water box in the CPU oracle (integrals on the host)."""
    from mopac_gpu_b200 import workloads as wl
    from oracle import scf_oracle as so
    nat, xyz, _ = wl.water_box(nwater)
    return so.make_system(nat, xyz)


def shift_value(args):
    """The SHIFT=n keyword of the timed SCF, or None for iter's default."""
    return None if (args.mode != "fast" or args.shift == "default") else float(args.shift)


def oracle_scf(s, mode: str, shift=None):
    """One complete oracle SCF from the standard guess, timed on the host:
    mode "fast" is the GPU arm's algorithm (pseudo-diagonalisation once newdg
    is set, Pulay, the SHIFT keyword, FP64 finish to max|dP| <= FINISH_DP),
    "plain" a full LAPACK eigensolve every iteration with cnvg (iter's
    default keywords).  Returns (result, seconds)."""
    from oracle import scf_oracle as so
    kw = dict(pseudo=True, pulay_on=True, finish_dp=FINISH_DP, shift_kw=shift) if mode == "fast" else {}
    t0 = time.perf_counter()
    r = so.iter_scf(s, **kw)
    return r, time.perf_counter() - t0


def warm_host(s, steps: int):
    """Untimed plain oracle steps (Fock build, eigensolve, density) to start
    the BLAS threads and page in the integrals."""
    import numpy as np
    from oracle import scf_oracle as so
    p = np.zeros(s.mpack)
    p[so.diag_index(s.norbs)] = s.pdiag
    for _ in range(steps):
        p, _, _ = so.roothaan_step(s, p)


def _cpu_one(mol):
    """One molecule's SCF with the CPU oracle (a pool worker's task)."""
    from oracle import scf_oracle as so
    r = so.iter_scf(so.make_system(mol[0], mol[1]))
    return r.escf


def batch_sample(n: int, nsample: int):
    """Indices of an evenly spaced sample of a batch of n molecules."""
    step = max(1, n // nsample)
    return list(range(0, n, step))[:nsample]


def cpu_batch_rate(mols, nsample: int, workers: int):
    """SCF/s of the CPU oracle over an evenly spaced sample of the molecules,
    `workers` processes (spawned) each running whole SCFs with one BLAS
    thread; the pool is warmed on one molecule per worker first.  Returns
    (rate, sample size, the sample's heats)."""
    import multiprocessing as mp
    sample = [mols[i] for i in batch_sample(len(mols), nsample)]
    old = os.environ.get("OPENBLAS_NUM_THREADS")
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    try:
        with mp.get_context("spawn").Pool(workers) as pool:
            pool.map(_cpu_one, mols[:workers], chunksize=1)
            t0 = time.perf_counter()
            heats = pool.map(_cpu_one, sample, chunksize=1)
            dt = time.perf_counter() - t0
    finally:
        if old is None:
            os.environ.pop("OPENBLAS_NUM_THREADS", None)
        else:
            os.environ["OPENBLAS_NUM_THREADS"] = old
    return len(sample) / dt, len(sample), heats


def run_batch(args, flush, L, ws=1, rank=0, dist=None):
    """The batched workload; returns the "batched" object on rank 0 (None on
    the others).  Under torchrun the job is args.batch molecules per GPU: a
    seeded list of args.batch * N alkanes split over the ranks by
    replicas.shard (cost n^3, balanced), no data-path collective; times are
    the max over ranks."""
    import numpy as np
    import torch
    from mopac_gpu_b200 import ScfContext, workloads
    from mopac_gpu_b200.batch import Batch
    from mopac_gpu_b200.replicas import max_over_ranks, shard
    mols_all = workloads.alkane_batch(args.batch * ws)
    costs = [float(np.where(np.asarray(m[0]) == 1, 1, 4).sum()) ** 3 for m in mols_all]
    mols = [mols_all[i] for i in shard(costs, rank, ws)]
    nat_tot = sum(len(m[0]) for m in mols_all)
    b = Batch(mols)
    # launch configuration chosen by the autotuner on this batch (untimed, like
    # the warm-up); the runs below replay the captured graph of that launch
    tuned_nb, tuned_per, tuned_ms = b.autotune()
    for _ in range(args.warmup):
        b.run()
    if dist is not None:
        dist.barrier()
    times = []
    l0 = L.mb_launch_count()
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        escf, niter, conv, t_ms = b.run()
        times.append(t_ms)
    launches = L.mb_launch_count() - l0
    t_ms = max_over_ranks(statistics.mean(times), dist, "cuda")
    b.set_phase_timing(True)
    b.run()
    ph = b.phase_cycles()
    b.set_phase_timing(False)
    tot = max(1, sum(ph.values()))
    b.close()
    # through the C ABI from host coordinates: create (H2D of the atoms,
    # integrals on the GPU), run, read the heats back, destroy
    e2e_t = []
    for step in range(args.steps + 1):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bb = Batch(mols)
        bb.set_config(tuned_nb, tuned_per)
        e2, _, _, _ = bb.run()
        bb.close()
        torch.cuda.synchronize()
        if step > 0:
            e2e_t.append(time.perf_counter() - t0)
    te = max_over_ranks(statistics.mean(e2e_t), dist, "cuda")
    if rank != 0:
        return None
    # the plain FP64 GPU path, one molecule at a time, on a sample (rank 0)
    nplain = min(32, len(mols))
    stepp = max(1, len(mols) // nplain)
    idx = list(range(0, len(mols), stepp))[:nplain]
    plain_ms, dhf = [], []
    for m in idx:
        ctx = ScfContext(*mols[m])
        ctx.hcore()
        ctx.run(pseudo=False, precision=0)
        r = ctx.run(pseudo=False, precision=0)
        plain_ms.append(r.t_total_ms)
        dhf.append(abs(r.escf - escf[m]))
        ctx.close()
    plain_rate = len(idx) / (sum(plain_ms) / 1000.0)
    out = {
        "workload": f"{len(mols_all)} {BATCH_WORKLOAD}" + (f", {args.batch} per GPU on {ws} GPUs" if ws > 1 else ""),
        "metric": "batched_scfs_per_s", "value": len(mols_all) / (t_ms / 1000.0), "unit": "SCF/s",
        "ms_per_step": t_ms, "steps": args.steps, "warmup": args.warmup, "dtype": "f64",
        "l2": "flushed between steps (256 MB write)",
        "atoms": nat_tot, "niter_mean": float(np.mean(niter)), "niter_max": int(niter.max()),
        "converged_fraction": float(conv.mean()),
        "gpu_launches_per_step": int(launches // max(1, args.steps)),
        "launch_config": {"back_transform_block": tuned_nb, "ctas_per_sm": tuned_per or "all that fit",
                          "autotune_best_ms": tuned_ms, "chosen_by": "mb_batch_autotune (6 configurations timed)",
                          "launch": "CUDA graph replay of the captured persistent launch"},
        "phase_share": {k: round(v / tot, 4) for k, v in ph.items()},
        "plain_fp64_gpu": {"value": plain_rate, "unit": "SCF/s", "sample": len(idx),
                           "mode": "one molecule at a time through mb_scf_run, full FP64 eigensolve every "
                                   "iteration, integrals resident",
                           "max_abs_dHf_vs_batched_kcal_mol": float(max(dhf))},
        "speedup_vs_plain_fp64": (len(mols_all) / (t_ms / 1000.0)) / plain_rate,
        "e2e": {"value": len(mols_all) / te, "unit": "SCF/s",
                "h2d_bytes_per_step": 28 * nat_tot + 4 * len(mols_all),
                "d2h_bytes_per_step": 8 * len(mols_all), "wall_s": te,
                "includes": "batch creation (atoms to the device, integrals on the GPU), SCFs, heats to the host"},
    }
    if not args.no_cpu_baseline:
        workers = os.cpu_count() or 1
        rate, ns, heats = cpu_batch_rate(mols, 8 * workers, workers)
        sidx = batch_sample(len(mols), 8 * workers)
        dh = np.abs(np.asarray(heats) - escf[sidx])
        out["cpu_baseline"] = {"value": rate, "unit": "SCF/s", "cores": workers, "kind": "port",
                               "sample": f"{ns} evenly spaced molecules of the batch, one whole oracle SCF per "
                                         f"task, {workers} spawned processes"}
        out["parity_vs_oracle"] = {"molecules": ns, "max_abs_dHf_kcal_mol": float(dh.max()),
                                   "mean_abs_dHf_kcal_mol": float(dh.mean()),
                                   "what": "heat of every sampled molecule in the timed batched launch against "
                                           "the oracle's complete SCF of the same molecule"}
    return out


def run_mozyme(nwater: int):
    """The MOZYME configuration: a seeded (H2O)_n box at 1.0 g/cm^3, CUTOFF=9
    (cutof1 = 81, cutof2 = 8.9^2, MOZYME/fillij.F90:108-112), FP64.  Time to
    converge = pair-block layout and hcore_for_MOZYME on the GPU + the
    starting LMOs + the whole SCF (mb_mz_scf_run), wall clock with the
    device synchronised; then the Fock build and the LMO density timed alone
    with CUDA events against their algorithmic bytes."""
    import numpy as np
    import torch
    from mopac_gpu_b200 import mozyme, workloads
    from mopac_gpu_b200._lib import lib
    nat, xyz, edge = workloads.water_box(nwater)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    L = mozyme.Layout(np.where(np.asarray(nat) == 1, 1, 4).astype(np.int32), xyz, 81.0, 8.9 ** 2)
    nat_d = torch.from_numpy(np.ascontiguousarray(nat, np.int32)).cuda()
    coord_d = torch.from_numpy(np.ascontiguousarray(xyz, np.float64)).cuda()
    h, w, enuclr = mozyme.hcore(L, nat_d, coord_d)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    iorbs, occ, vir = mozyme.water_lmos(nat, xyz, pad_atoms=400)
    Qo, Qv = mozyme.Lmos(L, occ), mozyme.Lmos(L, vir)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    atheat = lib().mb_atheat(len(nat), np.ascontiguousarray(nat, np.int32).ctypes.data)
    r = mozyme.scf_run(L, Qo, Qv, coord_d, w, h, enuclr, atheat)
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    peaks, src = _peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f = torch.empty_like(r["f"])
    for _ in range(2):
        mozyme.fock(L, coord_d, w, r["p"], h, out=f)
    ev0.record()
    for _ in range(5):
        mozyme.fock(L, coord_d, w, r["p"], h, out=f)
    ev1.record()
    torch.cuda.synchronize()
    ms_f = ev0.elapsed_time(ev1) / 5
    pd = torch.empty_like(r["p"])
    ev0.record()
    for _ in range(5):
        mozyme.density(L, Qo, 0, out=pd)
    ev1.record()
    torch.cuda.synchronize()
    ms_d = ev0.elapsed_time(ev1) / 5
    bytes_f = 8.0 * (L.s.nw + 3 * L.mpack)
    ncf_h, ic_h, _ = Qo.to_host()
    nncf_h = occ[1]
    used = sum(int(iorbs[ic_h[nncf_h[i]:nncf_h[i] + ncf_h[i]] - 1].sum()) for i in range(len(ncf_h)))
    bytes_d = 8.0 * (L.mpack + used)   # P written once, every used LMO coefficient read once
    out = {"workload": f"(H2O){nwater} water box, {len(nat)} atoms, {L.norbs} basis functions, MOZYME PM7 1SCF, "
                       f"CUTOFF=9, cell {edge:.1f} A, seeded random sequential insertion",
           "time_to_converge_s": t3 - t0, "layout_and_integrals_s": t1 - t0, "starting_lmos_s": t2 - t1,
           "scf_s": t3 - t2, "scf_device_ms": r["t_total_ms"], "niter": r["niter"], "converged": r["converged"],
           "escf_kcal_mol": r["escf"], "escf_per_water_kcal_mol": r["escf"] / nwater,
           "rejected_rotations": r["nrejected"], "stored_pairs": int(L.s.npairs), "mpack": L.mpack,
           "precision": "FP64 throughout (no mixed-precision MOZYME variant; the plain FP64 MOZYME path is this one)",
           "roofline_fock": {"kernel": "mz_fock (buildf/fock2z on the pair blocks)", "bound": "hbm",
                             "ms_per_launch": ms_f, "algorithmic_bytes": bytes_f,
                             "achieved": bytes_f / (ms_f * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                             "frac": bytes_f / (ms_f * 1e-3) / 1e9 / hbm, "peak_source": src},
           "roofline_density": {"kernel": "mz_density (density_for_MOZYME)", "bound": "hbm",
                                "ms_per_launch": ms_d, "algorithmic_bytes": bytes_d,
                                "achieved": bytes_d / (ms_d * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                                "frac": bytes_d / (ms_d * 1e-3) / 1e9 / hbm, "peak_source": src}}
    Qo.close()
    Qv.close()
    L.close()
    return out


def bench_config(args, edge: float) -> dict:
    """The workload description both arms print (the reference arm runs the
    same SCF algorithm on the host, in FP64 throughout)."""
    return {"workload": WORKLOAD, "mode": args.mode,
            "converger": "pulay" if (args.mode == "fast" and args.converger == "pulay") else "cnvg",
            "shift_keyword": "default (-80)" if shift_value(args) is None else shift_value(args),
            "finish_dp": FINISH_DP if args.precision == "split" else 0.0,
            "parallelism": "replicas x1" if args.gpus == 1 else f"replicas x{args.gpus}",
            "l2": "GPU: flushed between steps (256 MB write); W = 151 MB > L2",
            "cell_edge_A": round(edge, 3)}


def run_reference(args):
    """The reference arm: the CPU implementation of the same SCF (the oracle)
    on all host cores.  Its timed region is ONE complete SCF from the standard
    guess in the GPU arm's mode (fast: pseudo-diagonalisation, Pulay, finish
    to max|dP| <= FINISH_DP, FP64), because one SCF of the 3072-orbital box
    takes about a minute on the host; it is reported as --steps slices of
    that SCF (ms_per_step = SCF time / steps).  A complete plain-mode SCF
    (full eigensolve every iteration, cnvg) is timed beside it."""
    ws, rank, _ = dist_init()
    if rank != 0:
        return 0
    cores = os.cpu_count()
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(cores))
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    from mopac_gpu_b200 import workloads
    _, _, edge = workloads.water_box(args.nwater)
    s = oracle_system(args.nwater)
    warm_host(s, min(args.warmup, 2))
    r, t_scf = oracle_scf(s, args.mode, shift_value(args))
    rp, t_plain = oracle_scf(s, "plain") if args.mode == "fast" else (r, t_scf)
    val = 1.0 / t_scf
    mode_txt = ("pseudo-diagonalisation once newdg is set, Pulay, SHIFT keyword as in config, FP64 finish to "
                "max|dP| <= 1e-7, standard guess" if args.mode == "fast" else "full eigensolve every iteration, cnvg")
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "SCF/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_scf * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded water box, random sequential insertion)",
        "config": bench_config(args, edge),
        "guess": "standard diagonal guess (the reference has no learned guess)",
        "scf_wall_s": t_scf,
        "scf": {"escf_kcal_mol": r.escf, "niter": r.niter, "finish_iterations": r.n_finish, "converged": r.converged},
        "plain_mode": {"scf_wall_s": t_plain, "niter": rp.niter, "escf_kcal_mol": rp.escf,
                       "mode": "full LAPACK eigensolve every iteration, cnvg (iter's default)"},
        "cpu_baseline": {"value": val, "unit": "SCF/s", "cores": cores, "kind": "port",
                         "sample": f"one complete oracle SCF of the box ({mode_txt}; C Fock build and rotation "
                                   f"sweep, LAPACK dsyevd / BLAS on {cores} threads), timed whole; the line's "
                                   f"{args.steps} steps are equal slices of it"},
        "e2e": {"value": val, "unit": "SCF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if args.batch > 0:
        mols = workloads.alkane_batch(args.batch)
        rate, ns, _ = cpu_batch_rate(mols, 8 * cores, cores)
        line["batched"] = {"workload": f"{len(mols)} {BATCH_WORKLOAD}", "metric": "batched_scfs_per_s",
                           "value": rate, "unit": "SCF/s", "cores": cores, "kind": "port",
                           "sample": f"{ns} evenly spaced molecules of the batch, one whole oracle SCF per "
                                     f"task, {cores} spawned processes"}
    print(json.dumps(line), flush=True)
    return 0


def run_mine(args):
    import numpy as np
    import torch
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from mopac_gpu_b200 import ScfContext, workloads
    from mopac_gpu_b200._lib import lib
    L = lib()
    nat, xyz, edge = workloads.water_box(args.nwater)
    pseudo = args.mode == "fast"
    prec = 1 if args.precision == "split" else 0
    ctx = ScfContext(nat, xyz)
    ctx.hcore()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    from mopac_gpu_b200.guess import BOX_MODEL, GuessModel
    pul = pseudo and args.converger == "pulay"
    shift = shift_value(args)
    box_model = GuessModel(path=BOX_MODEL) if GuessModel.available(BOX_MODEL) else None
    model = box_model if args.guess == "learned" else None
    guess_note = "learned (atom-pair network trained on liquid-density boxes, prediction inside the timed step)" \
        if model else "standard diagonal guess" + (" (no trained blob found)" if args.guess == "learned" else "")

    def learned_step(c, mdl):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c.learned_guess(mdl)
        tp = (time.perf_counter() - t0) * 1e3
        rr = c.run(pseudo=pseudo, precision=prec, pulay=pul, guess=True, shift=shift)
        return rr, tp + rr.t_total_ms, tp

    def standard_step(c):
        rr = c.run(pseudo=pseudo, precision=prec, pulay=pul, shift=shift)
        return rr, rr.t_total_ms, 0.0

    def scf_step(c):
        """One step: (prediction +) SCF; returns (result, step ms, prediction ms)."""
        if model is None:
            return standard_step(c)
        return learned_step(c, model)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        r, _, _ = scf_step(ctx)
    # ---- timed region (device-resident inputs)
    clocks = ClockSampler(local)
    barrier()
    for kid in range(5):  # drop anything recorded before the timed region
        L.mb_kstats_read(kid, None, None)
    L.mb_kstats_enable(1)
    clocks.start()
    l0 = L.mb_launch_count()
    times, results, pred_ms = [], [], []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        r, tstep, tp = scf_step(ctx)
        times.append(tstep)
        pred_ms.append(tp)
        results.append(r)
    barrier()
    launches = L.mb_launch_count() - l0
    clk = clocks.stop()
    L.mb_kstats_enable(0)
    kst = {}
    for kid, name in enumerate(["tridiag_panel", "fock2", "density", "eigensolve", "pseudo_diag"]):
        cnt, tot = ctypes.c_longlong(0), ctypes.c_double(0.0)
        L.mb_kstats_read(kid, ctypes.byref(cnt), ctypes.byref(tot))
        kst[name] = {"launches": cnt.value, "total_ms": tot.value}
    from mopac_gpu_b200.replicas import max_over_ranks
    t_ms = max_over_ranks(statistics.mean(times), dist, "cuda")
    r = results[-1]
    # the timed SCF's density and orbital energies, for the oracle comparison
    p_fast = ctx.density()
    _, e_fast = ctx.vectors()
    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        h, w, enuc = ctx.get_hw()
        hp = torch.from_numpy(h).pin_memory()
        wp = torch.from_numpy(w).pin_memory()
        pout = torch.empty(ctx.mpack, dtype=torch.float64).pin_memory()
        e2e_t = []
        for step in range(args.steps + 1):
            flush.fill_(1.0)
            barrier()
            t0 = time.perf_counter()
            L.mb_ctx_set_hw(ctx._h, hp.data_ptr(), wp.data_ptr(), enuc)
            rr, _, _ = scf_step(ctx)
            L.mb_ctx_get_density(ctx._h, pout.data_ptr())
            torch.cuda.synchronize()
            if step > 0:
                e2e_t.append(time.perf_counter() - t0)
        te = max_over_ranks(statistics.mean(e2e_t), dist, "cuda")
        e2e = {"value": ws / te, "unit": "SCF/s", "h2d_bytes_per_step": 8 * (ctx.mpack + ctx.n2elec),
               "d2h_bytes_per_step": 8 * ctx.mpack, "scf_wall_s": te}
    # ---- rooflines: the dominant kernel (Householder panel) from the events
    # recorded on its stream inside the timed region, and the Fock build
    roof = panel_roofline(ctx, kst, eigh_sizes(ctx, results))
    roof_fock = fock_roofline(ctx)
    # ---- the plain FP64 GPU path on the same input (reference point of the
    # metric) and |dHf| of the timed SCF against FP64
    plain_ms = []
    r64 = None
    for i in range(3):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        rp = ctx.run(pseudo=False, precision=0)
        if i > 0:
            plain_ms.append(rp.t_total_ms)
        r64 = rp
    plain = {"scf_wall_s": statistics.mean(plain_ms) / 1000.0, "niter": r64.niter, "escf_kcal_mol": r64.escf,
             "mode": "full FP64 eigensolve every iteration, FP64 GEMMs, standard guess", "steps": len(plain_ms)}
    # the batched workload: every rank takes part (its collectives come before
    # any rank-0-only work)
    batched = run_batch(args, flush, L, ws, rank, dist) if args.batch > 0 else None
    # the learned guess on this box (the fast path from the network trained on
    # liquid-density boxes) and on held-out lattice clusters (its own case)
    guess_eval = None
    if rank == 0 and (box_model is not None or GuessModel.available()):
        guess_eval = {}
        if box_model is not None:
            # the same fast path from the other starting density
            lm = []
            for i in range(2):
                flush.fill_(1.0)
                rl, tl, tpl = standard_step(ctx) if model is not None else learned_step(ctx, box_model)
                lm.append(tl)
            guess_eval["standard_guess_fast_path" if model is not None else "learned_guess_fast_path"] = {
                "scf_wall_s_incl_prediction": lm[-1] / 1000.0, "prediction_ms": tpl, "niter": rl.niter,
                "full_diag": rl.n_full_diag, "pseudo_diag": rl.n_pseudo_diag, "finish_iterations": rl.n_finish,
                "abs_dHf_vs_fp64_kcal_mol": abs(rl.escf - r64.escf),
                "model": "guess_pm7_waterbox.npy (4000 seeded (H2O)16..64 boxes at 1.0 g/cm^3), one McWeeny step"}
        if GuessModel.available() and args.guess_sample > 0:
            from mopac_gpu_b200.guess import evaluate
            ev = evaluate(GuessModel(), n_clusters=args.guess_sample, nmin=32, nmax=128, seed=777)
            guess_eval["held_out_lattice"] = {
                "workload": "held-out (H2O)_n lattice clusters (as the 16-water case), n ~ U{32..128}, "
                            "PM7 1SCF, plain FP64 path, standard vs learned guess",
                "model": "guess_pm7_water.npy (20000 seeded (H2O)8..64 lattice clusters)",
                "clusters": ev.n_clusters, "niter_standard": ev.niter_std, "niter_learned": ev.niter_learned,
                "ms_standard": ev.ms_std, "ms_learned_incl_prediction": ev.ms_learned,
                "speedup": ev.ms_std / ev.ms_learned, "max_abs_dHf_kcal_mol": ev.max_dhf,
                "fallbacks": ev.n_fallback}
    mozyme_out = run_mozyme(args.mozyme) if (rank == 0 and args.mozyme > 0) else None
    cpu, parity = None, None
    if rank == 0 and not args.no_cpu_baseline:
        # the CPU oracle: one complete SCF of the same box in the same mode on
        # the host cores (the baseline), compared with the timed GPU SCF, and
        # the fixed-point certificate of the GPU density (three plain oracle
        # steps from it bound its distance to the self-consistent density)
        import numpy as np
        from oracle import scf_oracle as so
        cores = os.cpu_count()
        os.environ.setdefault("OPENBLAS_NUM_THREADS", str(cores))
        s_or = oracle_system(args.nwater)
        ro, t_or = oracle_scf(s_or, args.mode, shift)
        cpu = {"value": 1.0 / t_or, "unit": "SCF/s", "cores": cores, "kind": "port",
               "sample": "one complete oracle SCF of the box in the same mode (C Fock build and rotation sweep, "
                         f"LAPACK dsyevd / BLAS on {cores} threads), timed whole", "scf_wall_s": t_or,
               "niter": ro.niter}
        cert = so.fixed_point_certificate(s_or, p_fast, steps=3)
        parity = {
            "vs_oracle_same_mode": {"abs_dHf_kcal_mol": abs(r.escf - ro.escf),
                                    "max_abs_dP": float(np.abs(p_fast - ro.p).max()),
                                    "max_abs_deig_eV": float(np.abs(e_fast - ro.eigs).max()),
                                    "oracle_niter": ro.niter, "gpu_niter": r.niter,
                                    "what": "timed GPU SCF against the oracle's complete FP64 SCF of the box in the "
                                            "same mode (both finish to max|dP| <= 1e-7)"},
            "fixed_point_certificate": {"max_abs_dP_bound": cert["bound"], "rho": cert["rho"], "r": cert["r"],
                                        "max_abs_deig_eV": float(np.abs(e_fast - cert["eigs"]).max()),
                                        "abs_dHf_at_P_kcal_mol": abs(r.escf - cert["heat_at_p"]),
                                        "what": "three plain oracle steps from the GPU density: r_1/(1-rho) bounds "
                                                "max|P_gpu - P*|; eigenvalues of the oracle's F(P_gpu)"}}
    if rank == 0:
        line = {
            "metric": METRIC, "value": ws * 1000.0 / t_ms, "unit": "SCF/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == 0 else "f64+bf16x3",
            "data": "synthetic (seeded water box, random sequential insertion)",
            "config": bench_config(args, edge),
            "precision": args.precision,
            "scf_wall_s": t_ms / 1000.0,
            "guess": guess_note,
            "converger": "pulay" if pul else "cnvg",
            "guess_prediction_ms": statistics.mean(pred_ms),
            "learned_guess": guess_eval,
            "scf": {"escf_kcal_mol": r.escf, "niter": r.niter, "full_diag": r.n_full_diag,
                    "pseudo_diag": r.n_pseudo_diag, "split_iterations": r.n_split, "converged": r.converged,
                    "finish_iterations": r.n_finish, "last_max_abs_dP": r.dp,
                    "exit_split": r.exit_split, "exit_coupling_eV": r.exit_coupling,
                    "abs_dHf_vs_fp64_kcal_mol": abs(r.escf - r64.escf),
                    "phase_ms": {"fock": r.t_fock_ms, "diag": r.t_diag_ms, "density_cnvg": r.t_density_ms,
                                 "other": r.t_other_ms}},
            "plain_fp64_gpu": plain,
            "speedup_vs_plain_fp64": plain["scf_wall_s"] / (t_ms / 1000.0),
            "gpu_launches": int(launches),
            "gpu_launches_per_step": int(launches // max(1, args.steps)),
            "clocks": clk,
            "roofline": roof,
            "roofline_fock": roof_fock,
            "kernel_ms": {k: v["total_ms"] / max(1, args.steps) for k, v in kst.items()},
            "cpu_baseline": cpu,
            "parity_vs_oracle": parity,
            "e2e": e2e,
            "batched": batched,
            "mozyme": mozyme_out,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def eigh_sizes(ctx, results):
    """Orders of the eigensolves the timed SCFs ran: n for every full
    eigensolve, and nclose and n - nclose for an exit diagonalisation solved
    as the occupied and virtual blocks."""
    n, no = ctx.norbs, ctx.nclose
    sizes = []
    for r in results:
        sizes += [n] * r.n_full_diag
        if r.exit_split:
            sizes += [no, n - no]
    return sizes


def panel_roofline(ctx, kst, sizes):
    """Householder panel kernel: each reduced column reads its trailing
    matrix once for p = A22 v, 8*(m-j-1)^2 bytes for an eigensolve of order
    m; summed over the columns of every eigensolve of the timed region
    (sizes) and divided by the panel kernel's total time there."""
    st = kst["tridiag_panel"]
    if st["launches"] == 0 or not sizes:
        return None
    algo_total = sum(8.0 * (m - 1) * m * (2 * m - 1) / 6.0 for m in sizes)
    panels = sum((m - 2) // 32 + 1 for m in sizes if m > 1)
    ms = st["total_ms"] / st["launches"]
    peaks, src = _peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    ach = algo_total / (st["total_ms"] * 1e-3) / 1e9
    n = ctx.norbs
    return {"kernel": "tridiag_panel (Householder panel: column updates, reflectors, p = A22 v)",
            "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "traffic": PANEL_DRAM_BYTES * (algo_total / st["launches"]) / PANEL_ALGO_BYTES_3072,
            "ms_per_launch": ms, "algorithmic_bytes": algo_total / st["launches"],
            "launches": st["launches"], "launches_expected": panels, "eigensolve_orders": sorted(set(sizes)),
            "peak_source": src,
            "note": "algorithmic bytes: one read of the trailing matrix per column, over every eigensolve "
                    f"of the timed region (orders {sorted(set(sizes))}); the matrix ({8 * n * n / 1e6:.0f} MB "
                    "at the full order) is L2-resident, so DRAM traffic is far below it"}


# DRAM bytes (read + write) of the average tridiag_panel launch at n = 3072:
# an ncu capture of the first panel measured 249 MB against its 2.39 GB of
# algorithmic bytes (the matrix is L2-resident); scaled by algorithmic bytes to
# the average panel of the timed region.
PANEL_DRAM_BYTES = 8.39e7
PANEL_ALGO_BYTES_3072 = 8.0 * 3071 * 3072 * 6143 / 6.0 / 96


def fock_roofline(ctx):
    import torch
    from mopac_gpu_b200 import kernels as K
    from mopac_gpu_b200._lib import MbAtomsDev, lib
    import ctypes
    ptr = ctx.device_ptrs()
    at = MbAtomsDev()
    lib().mb_ctx_atoms_dev(ctx._h, ctypes.byref(at))
    mp = ctx.mpack
    f = torch.empty(mp, dtype=torch.float64, device="cuda")
    pa = torch.empty(mp, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # pa = p/2 as in the SCF
    p = ptr["p"]
    pt = torch.empty(mp, dtype=torch.float64, device="cuda")
    lib().mb_density_dev  # noqa: B018 (binding check)
    torch.cuda.synchronize()
    # copy the converged P out of the context into torch memory
    import numpy as np
    pt.copy_(torch.from_numpy(ctx.density()))
    pa.copy_(pt * 0.5)
    reps = 10
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    wsb = lib().mb_fock2_ws_bytes(len(ctx.nat))
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")

    def call():
        rc = lib().mb_fock2_ws(ctypes.byref(at), ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(ptr["h"]),
                               ctypes.c_void_p(pt.data_ptr()), ctypes.c_void_p(pa.data_ptr()),
                               ctypes.c_void_p(ptr["w"]), -20.0, 1, ctypes.c_void_p(ws.data_ptr()), wsb, stream)
        if rc != 0:
            raise RuntimeError(f"mb_fock2_ws failed ({rc})")

    for _ in range(2):
        call()
    ev0.record()
    for _ in range(reps):
        call()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / reps
    algo = 8.0 * (ctx.n2elec + 4 * mp)
    peaks, src = _peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    ach = algo / (ms * 1e-3) / 1e9
    return {"kernel": "fock2_pairs + fock2_fold (Fock build, fock2+fock1)", "bound": "hbm", "achieved": ach, "peak": peak,
            "unit": "GB/s", "frac": ach / peak, "traffic": None, "ms_per_launch": ms,
            "algorithmic_bytes": algo, "peak_source": src}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_mine(args)


if __name__ == "__main__":
    sys.exit(main())
