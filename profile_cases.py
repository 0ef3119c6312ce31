"""Per-kernel timing cases for the SCF rows, at the benchmark sizes.

  python profile_cases.py [case ...] [--reps R] [--out FILE]

Each case times one library entry point with CUDA events on the current
stream (warm-up first, L2 flushed by a 256 MB write before every timed
repetition) and prints one JSON line: the time per call, the algorithmic
bytes or flops of one call, the achieved rate and its fraction of the peak
it is bound by.  Peaks: HBM and BF16 from MEASURED_PEAKS.json at the
repository root (fallback 6650 GB/s, 1590 TFLOP/s); FP64 is measured here as
torch's float64 matmul at 8192^3 (cuBLAS DGEMM) because the pool's peak file
has no FP64 figure.

Cases (sizes of the benchmark configurations):
  fock2         Fock build, (H2O)512: 8 (n2elec + 4 mpack) bytes
  dcart         gradient (dcart), (H2O)512: four pair energies per atom pair
  helect, cnvg  energy and extrapolation, n = 3072: 24 mpack / 24 mpack + 8 n bytes
  density64     P = 2 C_o C_o^T FP64, n = 3072, k = 2048: n^2 k flops
  density_split same with the three-product BF16 split on tcgen05
  gemm64, gemm_split   3072^3 GEMM, 2 n^3 flops
  eigh          full eigensolve n = 3072 (the SCF's Fock matrix)
  eigh_cusolver the same matrix through torch.linalg.eigh (cuSOLVER's syevd),
                the library bar, beside this library's eigensolver
  eigh_rand     full eigensolve of a seeded random symmetric 3072 x 3072 matrix
                (no SCF before it: the case to run under a launch-list capture)
  pseudo_diag   Fmo + rotation sweep, n = 3072, k = 2048
  pulay         one Pulay step with a full 10-entry history, n = 3072
  batch         the batched SCF of seeded alkanes C3..C20 (--batch-n
                molecules, default 4096), one persistent launch, default
                launch configuration: SCF/s and FP64 flops of the reduction,
                back-transformation and density per iteration
  guess_features  learned guess: pair frames + descriptors of the (H2O)512 box
                (a warp per pair, three passes over the atoms)
  guess_forward   the five networks on every pair of the (H2O)512 box:
                2 rows (356*128 + 2*128*128 + 128*16) flops
  guess_train     one training step (forward, backward, Adam) of the O-H
                network on 2048 rows: 6 rows params flops
  guess_predict   the whole prediction into a context (mb_ctx_guess), (H2O)512
  mz_scf_split  the MOZYME SCF of the (H2O)4096 box (CUTOFF=9, the bench's
                starting LMOs) through the host loop with every step
                synchronised and timed: seconds per step over the SCF
  mz_density, mz_helecz, mz_cnvgz, mz_fock, mz_diagg1, mz_diagg2
                MOZYME blocks, (H2O)4096, 9 A cutoff, synthetic unit LMOs
                (occupied over 4 A, virtual over 3.2 A, two spare atom slots),
                seeded random integrals for the Fock build (timing only)
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys

import numpy as np
import torch

from mopac_gpu_b200 import kernels, mozyme, workloads
from mopac_gpu_b200._lib import MbAtomsDev, check, lib
from mopac_gpu_b200.scf import ScfContext

ROOT = os.path.dirname(os.path.abspath(__file__))


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


_flush = None


def flush_l2():
    global _flush
    if _flush is None:
        _flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    _flush.fill_(1.0)


def timed(fn, reps: int, warm: int = 2, setup=None):
    for _ in range(warm):
        if setup:
            setup()
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        if setup:
            setup()
        flush_l2()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def s():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


_fp64_peak = None


def fp64_peak_tflops():
    global _fp64_peak
    if _fp64_peak is None:
        a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
        b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
        ms = timed(lambda: torch.matmul(a, b), 3, 1)
        _fp64_peak = 2 * 8192 ** 3 / (ms * 1e-3) / 1e12
        del a, b
    return _fp64_peak


def line(case, ms, work, unit, bound, peak, peak_src, **extra):
    scale = 1e9 if unit == "GB/s" else 1e12
    ach = work / (ms * 1e-3) / scale
    d = {"case": case, "ms": round(ms, 4), "achieved": round(ach, 2), "unit": unit, "bound": bound,
         "peak": round(peak, 1), "frac": round(ach / peak, 4), "peak_source": peak_src,
         "work_per_call": work}
    d.update(extra)
    return d


class C1:
    """(H2O)512 context converged once, plus device copies for the kernels."""

    def __init__(self):
        nat, xyz, _ = workloads.water_box(512)
        self.ctx = ScfContext(nat, xyz)
        self.ctx.hcore()
        self.ctx.run(pseudo=True)
        self.n = self.ctx.norbs
        self.k = self.ctx.nclose
        self.mpack = self.ctx.mpack
        ptr = self.ctx.device_ptrs()
        self.ptr = ptr
        mp, n = self.mpack, self.n

        def wrap(addr, count):
            # torch views of library-owned device memory through __cuda_array_interface__
            class _A:
                __cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (addr, False),
                                            "version": 3, "strides": None}
            return torch.as_tensor(_A(), device="cuda")

        self.h = wrap(ptr["h"], mp)
        self.w = wrap(ptr["w"], self.ctx.n2elec)
        self.f = wrap(ptr["f"], mp)
        self.p = wrap(ptr["p"], mp)
        self.c = wrap(ptr["c"], n * n)
        self.eigs = wrap(ptr["eigs"], n)
        self.pa = (self.p * 0.5).contiguous()
        self.atoms = MbAtomsDev()
        check(lib().mb_ctx_atoms_dev(self.ctx._h, ctypes.byref(self.atoms)))


def mz_scf_split(nwater: int = 4096) -> dict:
    """Per-step seconds of mozyme.iter_for_mozyme on the (H2O)_n box, each
    step wrapped in torch.cuda.synchronize() (the loop mb_mz_scf_run runs in
    C, composed of the same entry points)."""
    import collections
    import time
    from mopac_gpu_b200 import mozyme as mz
    T = collections.defaultdict(float)

    def timed(name, fn):
        def w(*a, **k):
            torch.cuda.synchronize()
            t = time.perf_counter()
            r = fn(*a, **k)
            torch.cuda.synchronize()
            T[name] += time.perf_counter() - t
            return r
        return w

    L_ = lib()
    saved = []
    for nm in ("mb_mz_tidy_dev", "mb_mz_check_dev", "mb_mz_eimp_dev", "mb_mz_hbonds_dev"):
        saved.append((L_, nm, getattr(L_, nm)))
        setattr(L_, nm, timed(nm.replace("mb_mz_", "").replace("_dev", ""), getattr(L_, nm)))
    for nm in ("diagg2", "density", "cnvgz", "fock", "helecz"):
        saved.append((mz, nm, getattr(mz, nm)))
        setattr(mz, nm, timed(nm, getattr(mz, nm)))

    def refresh_dev(self):
        check(lib().mb_mz_lmos_refresh_dev(self.numat, ctypes.c_void_p(self.layout_iorbs), ctypes.byref(self.s), None))

    saved.append((mz.Lmos, "refresh", mz.Lmos.refresh))
    mz.Lmos.refresh = timed("lmo_index_refresh", refresh_dev)
    base = mz.Diagg1

    class TimedDiagg1(base):
        def __call__(self, *a, **k):
            return timed("diagg1", super().__call__)(*a, **k)

    saved.append((mz, "Diagg1", base))
    mz.Diagg1 = TimedDiagg1
    try:
        nat, xyz, _ = workloads.water_box(nwater)
        L = mz.Layout(np.where(np.asarray(nat) == 1, 1, 4).astype(np.int32), xyz, 81.0, 8.9 ** 2)
        nat_d = torch.from_numpy(np.ascontiguousarray(nat, np.int32)).cuda()
        coord_d = torch.from_numpy(np.ascontiguousarray(xyz, np.float64)).cuda()
        h, w, enuclr = mz.hcore(L, nat_d, coord_d)
        iorbs, occ, vir = mz.water_lmos(nat, xyz, pad_atoms=400)
        Qo, Qv = mz.Lmos(L, occ), mz.Lmos(L, vir)
        Qo.layout_iorbs = Qv.layout_iorbs = L.s.iorbs
        atheat = lib().mb_atheat(len(nat), np.ascontiguousarray(nat, np.int32).ctypes.data)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = mz.iter_for_mozyme(L, Qo, Qv, coord_d, w, h, enuclr, atheat)
        torch.cuda.synchronize()
        total = time.perf_counter() - t0
    finally:
        for obj, nm, v in saved:
            setattr(obj, nm, v)
    return {"case": "mz_scf_split", "total_s": round(total, 3), "niter": r["niter"],
            "escf_per_water_kcal_mol": r["escf"] / nwater,
            "steps_s": {k: round(v, 3) for k, v in sorted(T.items(), key=lambda x: -x[1])},
            "config": f"(H2O){nwater} box, CUTOFF=9, host loop with synchronised steps"}


def run_cases(names, reps):
    L = lib()
    pk = peaks()
    out = []
    hbm, bf16, src = pk["hbm_gbs"], pk["bf16_tflops"], pk["source"]
    need_c1 = any(c in names for c in ("fock2", "dcart", "helect", "cnvg", "density64", "density_split", "eigh", "eigh_cusolver",
                                       "pseudo_diag", "pulay"))
    c1 = C1() if need_c1 else None
    fp64 = fp64_peak_tflops() if any(c in names for c in ("density64", "gemm64", "eigh")) else None
    if "fock2" in names:
        f = c1.f.clone()
        wsb = L.mb_fock2_ws_bytes(len(c1.ctx.nat))
        ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
        ms = timed(lambda: check(L.mb_fock2_ws(ctypes.byref(c1.atoms), vp(f), vp(c1.h), vp(c1.p), vp(c1.pa),
                                               vp(c1.w), 0.0, 0, vp(ws), wsb, s())), reps)
        out.append(line("fock2", ms, 8 * (c1.ctx.n2elec + 4 * c1.mpack), "GB/s", "hbm", hbm, src,
                        config="(H2O)512, n = 3072"))
    if "mz_scf_split" in names:
        out.append(mz_scf_split())
    if "dcart" in names:
        wsb = L.mb_dcart_ws_bytes(len(c1.ctx.nat))
        ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
        g = torch.empty(3 * len(c1.ctx.nat), dtype=torch.float64, device="cuda")
        nat_d = torch.as_tensor(np.asarray(c1.ctx.nat, np.int32), device="cuda")
        xyz_d = torch.as_tensor(np.asarray(c1.ctx.coord, np.float64).ravel(), device="cuda")
        ms = timed(lambda: check(L.mb_dcart_dev(vp(nat_d), vp(xyz_d), ctypes.byref(c1.atoms), len(c1.ctx.nat),
                                                vp(c1.p), vp(g), vp(ws), wsb, s())), reps)
        npair = len(c1.ctx.nat) * (len(c1.ctx.nat) - 1) // 2
        out.append({"case": "dcart", "ms": round(ms, 4), "atom_pairs": npair,
                    "pair_energies_per_s": 4 * npair / (ms * 1e-3),
                    "config": "(H2O)512 gradient: four pair energies (integrals, Coulomb, exchange, "
                              "core-core) per atom pair, then the per-atom ordered sums"})
    if "helect" in names:
        o = torch.zeros(1, dtype=torch.float64, device="cuda")
        ms = timed(lambda: check(L.mb_helect_dev(c1.n, vp(c1.pa), vp(c1.h), vp(c1.f), vp(o), s())), reps)
        out.append(line("helect", ms, 24 * c1.mpack, "GB/s", "hbm", hbm, src, config="n = 3072"))
    if "cnvg" in names:
        pn, po, p1 = c1.p.clone(), c1.p.clone() * 0.999, torch.ones(c1.n, dtype=torch.float64, device="cuda")
        pl = torch.zeros(1, dtype=torch.float64, device="cuda")
        ms = timed(lambda: check(L.mb_cnvg_dev(c1.n, vp(pn), vp(po), vp(p1), 5, vp(pl), s())), reps)
        out.append(line("cnvg", ms, 24 * c1.mpack + 8 * c1.n, "GB/s", "hbm", hbm, src, config="n = 3072"))
    if "density64" in names or "density_split" in names:
        ct = c1.c.view(c1.n, c1.n)  # row-major view of column-major C: row index = column of C
        cc = ct.t()
        if "density64" in names:
            ms = timed(lambda: kernels.density(cc, c1.k), reps)
            out.append(line("density64", ms, c1.n ** 2 * c1.k, "TFLOP/s", "fp64", fp64, "cuBLAS DGEMM here",
                            config="n = 3072, k = 2048"))
        if "density_split" in names:
            ms = timed(lambda: kernels.density_split(cc, c1.k), reps)
            out.append(line("density_split", ms, c1.n ** 2 * c1.k, "TFLOP/s", "tensor", bf16, src,
                            config="n = 3072, k = 2048", note="algorithmic n^2 k against the BF16 peak; the "
                            "tensor pipe does 3x that (three BF16 products) on the lower tiles only"))
    if "gemm64" in names or "gemm_split" in names:
        n = 3072
        a = torch.randn(n, n, dtype=torch.float64, device="cuda")
        b = torch.randn(n, n, dtype=torch.float64, device="cuda")
        cm = torch.empty(n, n, dtype=torch.float64, device="cuda")
        if "gemm64" in names:
            ms = timed(lambda: check(L.mb_dgemm_dev(b"N", b"N", n, n, n, 1.0, vp(a), n, vp(b), n, 0.0, vp(cm), n,
                                                    s())), reps)
            out.append(line("gemm64", ms, 2 * n ** 3, "TFLOP/s", "fp64", fp64, "cuBLAS DGEMM here", config="3072^3"))
        if "gemm_split" in names:
            nb = int(L.mb_gemm_split_ws_bytes(n, n, n))
            buf, ws = kernels._aligned_ws(nb, "cuda")
            err = torch.zeros(1, dtype=torch.int32, device="cuda")
            ms = timed(lambda: check(L.mb_gemm_split_ws(b"N", b"N", n, n, n, 1.0, vp(a), n, vp(b), n, 0.0, vp(cm),
                                                        n, ws, nb, vp(err), s())), reps)
            assert int(err.item()) == 0
            out.append(line("gemm_split", ms, 2 * n ** 3, "TFLOP/s", "tensor", bf16, src, config="3072^3",
                            note="algorithmic 2 n^3 against the BF16 peak (the pipe does 3x)"))
    if "eigh" in names:
        fpk = c1.f.clone()
        work = fpk.clone()
        cv = torch.empty(c1.n * c1.n, dtype=torch.float64, device="cuda")
        ev = torch.empty(c1.n, dtype=torch.float64, device="cuda")
        nb = int(L.mb_eigh_ws_bytes(c1.n))
        buf, ws = kernels._aligned_ws(nb, "cuda", 256)
        st = torch.zeros(4, dtype=torch.int32, device="cuda")
        ms = timed(lambda: check(L.mb_eigh_ws(c1.n, vp(work), 1, vp(cv), vp(ev), ws, vp(st), s())),
                   max(2, reps // 2), setup=lambda: work.copy_(fpk))
        assert int(st[0].item()) == 0
        out.append(line("eigh", ms, 4.5 * c1.n ** 3, "TFLOP/s", "fp64", fp64, "cuBLAS DGEMM here",
                        config="n = 3072 Fock matrix of (H2O)512", note="4.5 n^3 flop convention of the "
                        "reference's gpu_bench"))
    if "eigh_cusolver" in names:
        # the library bar: cuSOLVER's dsyevd through torch.linalg.eigh on the
        # same Fock matrix (unpacked, with the reference's perturbation)
        fpk = c1.f.clone()
        work = fpk.clone()
        cv = torch.empty(c1.n * c1.n, dtype=torch.float64, device="cuda")
        ev = torch.empty(c1.n, dtype=torch.float64, device="cuda")
        nb = int(L.mb_eigh_ws_bytes(c1.n))
        buf, ws = kernels._aligned_ws(nb, "cuda", 256)
        st = torch.zeros(4, dtype=torch.int32, device="cuda")
        ms_ours = timed(lambda: check(L.mb_eigh_ws(c1.n, vp(work), 1, vp(cv), vp(ev), ws, vp(st), s())),
                        max(2, reps // 2), setup=lambda: work.copy_(fpk))
        a = torch.zeros(c1.n, c1.n, dtype=torch.float64, device="cuda")
        rr, cc = torch.tril_indices(c1.n, c1.n, device="cuda")
        a[rr, cc] = fpk
        a[cc, rr] = fpk
        a.diagonal().add_(torch.arange(1, c1.n + 1, dtype=torch.float64, device="cuda") * 1e-10)
        ms_lib = timed(lambda: torch.linalg.eigh(a), max(2, reps // 2))
        w_lib = torch.linalg.eigh(a)[0]
        out.append(line("eigh_cusolver", ms_lib, 4.5 * c1.n ** 3, "TFLOP/s", "fp64", fp64_peak_tflops(),
                        "cuBLAS DGEMM here", config="n = 3072 Fock matrix of (H2O)512",
                        ours_ms=ms_ours, library="torch.linalg.eigh (cuSOLVER syevd)",
                        max_abs_eig_diff=float((w_lib - ev).abs().max().item())))
    if "eigh_rand" in names:
        n = 3072
        rng = np.random.default_rng(0)
        a = rng.normal(size=(n, n))
        rr, cc = np.tril_indices(n)
        fpk = torch.from_numpy(np.ascontiguousarray((0.5 * (a + a.T))[rr, cc])).cuda()
        work = fpk.clone()
        cv = torch.empty(n * n, dtype=torch.float64, device="cuda")
        ev = torch.empty(n, dtype=torch.float64, device="cuda")
        nb = int(L.mb_eigh_ws_bytes(n))
        buf, ws = kernels._aligned_ws(nb, "cuda", 256)
        st = torch.zeros(4, dtype=torch.int32, device="cuda")
        ms = timed(lambda: check(L.mb_eigh_ws(n, vp(work), 1, vp(cv), vp(ev), ws, vp(st), s())), reps, warm=1,
                   setup=lambda: work.copy_(fpk))
        assert int(st[0].item()) == 0
        out.append(line("eigh_rand", ms, 4.5 * n ** 3, "TFLOP/s", "fp64", fp64_peak_tflops(), "cuBLAS DGEMM here",
                        config="n = 3072 seeded random symmetric"))
    if "pseudo_diag" in names:
        cv = c1.c.clone()
        nrot = ctypes.c_longlong(0)
        # the converged F has no rotations left; a seeded perturbation of F
        # (1e-3 eV per element) gives the sweep the work of an SCF iteration
        gen = torch.Generator(device="cuda").manual_seed(7)
        fpert = c1.f + 1e-3 * torch.randn(c1.f.shape, dtype=torch.float64, device="cuda", generator=gen)
        ms = timed(lambda: check(L.mb_pseudo_diag_dev(c1.n, c1.k, vp(fpert), vp(cv), vp(c1.eigs), ctypes.byref(nrot),
                                                      s())), reps, setup=lambda: cv.copy_(c1.c))
        v = c1.n - c1.k
        fl = 2 * c1.n * c1.n * v + 2 * v * c1.k * c1.n
        out.append(line("pseudo_diag", ms, fl, "TFLOP/s", "fp64", fp64_peak_tflops(), "cuBLAS DGEMM here",
                        config="n = 3072, k = 2048", rotations=int(nrot.value),
                        note="flops of the two Fmo GEMMs; the rotation sweep moves 32 n bytes per rotation"))
    if "pulay" in names:
        pu = kernels.Pulay(c1.n)
        f = c1.f.clone()
        for _ in range(10):
            pu.step(f, c1.pa)
        ms = timed(lambda: pu.step(f, c1.pa), reps, setup=lambda: f.copy_(c1.f))
        out.append(line("pulay", ms, 2 * c1.n ** 3, "TFLOP/s", "fp64", fp64_peak_tflops(), "cuBLAS DGEMM here",
                        config="n = 3072, 10 stored entries",
                        note="dominated by the n^3 commutator GEMM; history traffic 2 x 10 x 8 mpack bytes"))
    if any(c.startswith("mz_") for c in names):
        nat, xyz, _ = workloads.water_box(4096)
        iorbs, lmos = workloads.mozyme_lmos(nat, xyz, radius=4.0)
        c1c, c2c = 9.0 ** 2 + 1e-4, 9.0 ** 2
        lay = mozyme.Layout(iorbs, xyz, c1c, c2c)
        q = mozyme.Lmos(lay, lmos)
        mp = lay.mpack
        cfg = f"(H2O)4096, 9 A cutoff: mpack = {mp}, {len(lmos[0])} LMOs, {len(lmos[4])} coefficients"
        p = torch.empty(mp, dtype=torch.float64, device="cuda")
        mozyme.density(lay, q, 0, None, p)
        if "mz_density" in names:
            ms = timed(lambda: mozyme.density(lay, q, 0, None, p), reps)
            out.append(line("mz_density", ms, 8 * mp + 8 * len(lmos[4]), "GB/s", "hbm", hbm, src, config=cfg,
                            note="P written once and the coefficients read once; the merges re-read "
                            "coefficients from L2"))
        rng = np.random.default_rng(0)
        h = torch.from_numpy(rng.normal(size=mp)).cuda()
        f = torch.from_numpy(rng.normal(size=mp)).cuda()
        if "mz_helecz" in names:
            ws = torch.empty(int(L.mb_mz_helecz_ws_bytes()) // 8 + 1, dtype=torch.float64, device="cuda")
            o = torch.zeros(1, dtype=torch.float64, device="cuda")
            ms = timed(lambda: check(L.mb_mz_helecz_ws(mp, lay.norbs, vp(lay.idiag), vp(p), vp(h), vp(f), vp(o),
                                                       vp(ws), s())), reps)
            out.append(line("mz_helecz", ms, 24 * mp, "GB/s", "hbm", hbm, src, config=cfg))
        if "mz_cnvgz" in names:
            n = lay.norbs
            pn, po = p.clone(), p.clone() * 0.999
            p1, p2, p3 = (torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3))
            pm = torch.zeros(1, dtype=torch.float64, device="cuda")
            ws = torch.empty(32, dtype=torch.float64, device="cuda")
            ms = timed(lambda: check(L.mb_mz_cnvgz_ws(n, mp, vp(pn), vp(po), vp(p1), vp(p2), vp(p3), 6,
                                                      vp(lay.idiag), 1, vp(pm), vp(ws), s())), reps,
                       setup=lambda: (pn.copy_(p), po.copy_(p * 0.999)))
            out.append(line("mz_cnvgz", ms, 8 * 5 * mp + 8 * 5 * n, "GB/s", "hbm", hbm, src, config=cfg,
                            note="niter = 6: gather + max, one-thread factor, extrapolation, damping, copy"))
        if "mz_fock" in names:
            nw = int(lay.s.nw)
            wv = torch.from_numpy(rng.normal(size=nw) * 0.1).cuda()
            xyz_d = torch.from_numpy(np.ascontiguousarray(xyz, np.float64)).cuda()
            fo = torch.empty(mp, dtype=torch.float64, device="cuda")
            ms = timed(lambda: mozyme.fock(lay, xyz_d, wv, p, h, fo), reps)
            out.append(line("mz_fock", ms, 8 * nw + 8 * 3 * mp, "GB/s", "hbm", hbm, src, config=cfg,
                            note=f"stored-pair integrals ({nw} values) read once, P and H read, F written; "
                                 "every atom also scans all others for the point-charge terms"))
        if "mz_diagg1" in names or "mz_diagg2" in names:
            _, occ = workloads.mozyme_lmos(nat, xyz, radius=4.0, seed=3, per_heavy=4, pad_atoms=2)
            _, vir = workloads.mozyme_lmos(nat, xyz, radius=3.2, seed=4, per_heavy=2, pad_atoms=2)
            qo, qv = mozyme.Lmos(lay, occ), mozyme.Lmos(lay, vir)
            pz = mozyme.density(lay, qo, 0)
            cap = 300 * lay.norbs
            d1 = mozyme.Diagg1(lay, qo, qv, cap)
            if "mz_diagg1" in names:
                ms = timed(lambda: d1(h, pz, 0), max(2, reps // 2))
                out.append(line("mz_diagg1", ms, 8 * (mp + len(occ[4]) + len(vir[4])), "GB/s", "latency", hbm, src,
                                config=cfg, list_entries=int(d1.nij),
                                note="rebuild of the interaction list (idiagg = 0) over all occupied x virtual "
                                     "pairs; bytes = F once plus the coefficients once"))
            if "mz_diagg2" in names:
                d1(h, pz, 0)
                nrejct = np.zeros(2, np.int32)
                ctl = [1.0, 0.0, 1e-13, float(d1.state[3]), 50 * np.sqrt(1e-39)]
                t0 = torch.cuda.Event(enable_timing=True)
                t1 = torch.cuda.Event(enable_timing=True)
                flush_l2()
                t0.record()
                sb, nrej = mozyme.diagg2(lay, qo, qv, d1, 0, ctl, nrejct)
                t1.record()
                torch.cuda.synchronize()
                ms = t0.elapsed_time(t1)
                out.append(line("mz_diagg2", ms, 32 * int(d1.nij) * 4 * 20, "GB/s", "latency", hbm, src, config=cfg,
                                rotations=int(d1.nij), rejected=int(nrej),
                                note="one pass over the list in dependency levels (host level build included); "
                                     "bytes: nominal 2 LMOs x 20 atoms x 4 orbitals read+write per rotation"))
            qo.close()
            qv.close()
        q.close()
        lay.close()
    if any(c.startswith("guess_") for c in names):
        out += guess_cases(names, reps, bf16, src)
    if "batch" in names:
        out += batch_case(reps)
    if c1 is not None:
        c1.ctx.close()
    return out


BATCH_N = 4096


def batch_case(reps):
    from mopac_gpu_b200.batch import Batch
    mols = workloads.alkane_batch(BATCH_N)
    b = Batch(mols)
    res = {}

    def run():
        res["r"] = b.run()
    ms = timed(run, reps)
    escf, niter, conv, _ = res["r"]
    flops = 0.0
    for m, (nat, _) in enumerate(mols):
        n = int(np.where(np.asarray(nat) == 1, 1, 4).sum())
        k = n // 2  # alkanes: valence electrons = basis functions
        flops += niter[m] * (4.0 * n ** 3 / 3.0 + 3.0 * n * n * k)
    fp64 = fp64_peak_tflops()
    nb, grid = b.config()
    b.close()
    return [line("batch", ms, flops, "TFLOP/s", "FP64 latency (barriers, dependent chains)", fp64, "measured here",
                 molecules=len(mols), scf_per_s=len(mols) / (ms * 1e-3), niter_mean=float(np.mean(niter)),
                 converged=bool(conv.all()), back_transform_block=nb, grid=grid,
                 note="flops: per iteration 4n^3/3 (reduction) + 2n^2 nocc (back-transformation) + "
                      "n^2 nocc (density); nocc = electrons/2 of an alkane = n/2")]


def guess_cases(names, reps, bf16, src):
    """Learned-guess kernels on the (H2O)512 box (an untrained, seeded blob:
    the timing does not depend on the weights)."""
    from mopac_gpu_b200 import guess as G
    L = lib()
    out = []
    nat, xyz, _ = workloads.water_box(512)
    ps = G.PairSet(nat, xyz)
    model = G.GuessModel(G.init_blob(0)) if not G.GuessModel.available() else G.GuessModel()
    DIN_BYTES = G.DIN + 18  # floats of descriptors + the frame's nine doubles

    def hbm_peak():
        return peaks()["hbm_gbs"]
    if "guess_features" in names:
        ms = timed(lambda: check(L.mb_guess_features_dev(ps.numat, ps.nat.data_ptr(), ps.xyz.data_ptr(), ps.n,
                                                         ps.pf.data_ptr(), ps.ps.data_ptr(), ps.feat.data_ptr(),
                                                         ps.frames.data_ptr(), ps.ws.data_ptr(), s())), reps)
        work = 4.0 * ps.n * DIN_BYTES  # descriptors written (FP32) + frames
        out.append(line("guess_features", ms, work, "GB/s", "FP64 issue / latency", hbm_peak(), src,
                        pairs=ps.n, atoms=ps.numat,
                        note="work = descriptor bytes written; the kernel is FP64-issue bound "
                             "(neighbour lists within 6 A, all atoms for the frame and the long-range terms)"))
    xs, ys, wss = [], [], []
    for t in range(G.NTYPES):
        a, b = ps.offsets[t], ps.offsets[t + 1]
        x = torch.empty((b - a, G.DIN), dtype=torch.int16, device="cuda")
        check(L.mb_guess_normalize_dev(model.handle, t, b - a, ps.feat[a:b].data_ptr(), x.data_ptr(), s()))
        xs.append(x)
        ys.append(torch.empty((b - a, G.DOUT), dtype=torch.float32, device="cuda"))
        wss.append(torch.empty(2 * (b - a) * G.HID, dtype=torch.int16, device="cuda"))
    rows = ps.n
    flops_row = 2.0 * (G.DIN * G.HID + 2 * G.HID * G.HID + G.HID * G.DOUT)
    if "guess_forward" in names:
        def fwd():
            for t in range(G.NTYPES):
                if xs[t].shape[0]:
                    check(L.mb_guess_forward_dev(model.handle, t, xs[t].shape[0], xs[t].data_ptr(),
                                                 ys[t].data_ptr(), wss[t].data_ptr(), s()))
        ms = timed(fwd, reps)
        out.append(line("guess_forward", ms, flops_row * rows, "TFLOP/s", "BF16 tensor (mma.sync)", bf16, src,
                        rows=rows, launches=4 * G.NTYPES))
    if "guess_train" in names:
        n = 2048
        tr = G.Trainer(G.init_blob(1), n)
        x = xs[3][:n].contiguous()
        yt = torch.randn((n, G.DOUT), device="cuda")
        ms = timed(lambda: tr.step(3, x, yt, 1e-4), reps)
        params = G.DIN * G.HID + G.HID + 2 * (G.HID * G.HID + G.HID) + G.HID * G.DOUT + G.DOUT
        out.append(line("guess_train", ms, 6.0 * n * params, "TFLOP/s", "BF16 tensor (mma.sync) / launches", bf16,
                        src, rows=n, note="forward 2, backward 4 flops per row and parameter; 13 launches"))
        tr.close()
    if "guess_predict" in names:
        ctx = ScfContext(nat, xyz)
        ms = timed(lambda: ctx.learned_guess(model), reps)
        out.append(line("guess_predict", ms, flops_row * rows, "TFLOP/s", "descriptors (FP64) + launches", bf16, src,
                        pairs=rows, note="pairs, descriptors, five networks, assembly, with allocations"))
        ctx.close()
    model.close()
    return out


ALL = ["fock2", "dcart", "helect", "cnvg", "density64", "density_split", "gemm64", "gemm_split", "eigh", "eigh_cusolver", "eigh_rand",
       "pseudo_diag",
       "pulay", "mz_density", "mz_helecz", "mz_cnvgz", "mz_fock", "mz_diagg1", "mz_diagg2",
       "guess_features", "guess_forward", "guess_train", "guess_predict", "batch"]


EXTRA = ["mz_scf_split"]  # not in the default run (a whole MOZYME SCF)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="*", default=ALL)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--out", default=None)
    ap.add_argument("--batch-n", type=int, default=4096)
    a = ap.parse_args(argv)
    global BATCH_N
    BATCH_N = a.batch_n
    bad = [c for c in a.cases if c not in ALL + EXTRA]
    if bad:
        raise SystemExit(f"unknown cases {bad}; known: {ALL + EXTRA}")
    res = run_cases(a.cases, a.reps)
    for d in res:
        print(json.dumps(d), flush=True)
    if a.out:
        with open(a.out, "w") as fh:
            for d in res:
                fh.write(json.dumps(d) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
