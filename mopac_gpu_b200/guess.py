"""Learned initial guess: the atom-pair network, its training and its evaluation.

The network and every step around it run in libmopac_b200.so (csrc/guess.cu):
pair lists, frames and descriptors, the BF16 tensor-core forward and backward
passes, Adam, and the assembly of the predicted blocks into the packed
density.  This module is the host side: it loads a trained parameter blob,
generates training data with the plain FP64 SCF (``ScfContext.run``), drives
the trainer and compares SCFs started from the network against the standard
guess.  PyTorch only holds device buffers here (the data set, minibatch
gathers); no arithmetic of the network runs in it.

The reference has no learned guess: it starts iter from the diagonal guess
(moldat.F90:731-760) or from an OLDENS density (SCF/iter.F90:151-158); the
predicted density enters the same way as the latter, so the converged heat is
the SCF's own.
"""
from __future__ import annotations

import ctypes
import math
import os
import time
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib
from .scf import ScfContext
from . import workloads

DIN, HID, DOUT, NTYPES, PER_TYPE = 356, 128, 16, 5, 81528
NOUT = (10, 1, 16, 4, 1)
TYPE_NAMES = ("O own", "H own", "O-O", "O-H", "H-H")
RPAIR = 6.0
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "data", "guess_pm7_water.npy")          # lattice clusters
BOX_MODEL = os.path.join(HERE, "data", "guess_pm7_waterbox.npy")           # liquid-density boxes


def make_cluster(kind: str, nw: int, seed: int):
    """(nat, xyz) of a seeded (H2O)_nw: "lattice" (cubic lattice, 2.9 A, the
    16-water case's generator) or "box" (random sequential insertion at
    1.0 g/cm^3, the 512-water box's generator)."""
    if kind == "lattice":
        return workloads.water_lattice(nw, seed=seed)
    if kind == "box":
        nat, xyz, _ = workloads.water_box(nw, seed=seed)
        return nat, xyz
    raise ValueError(kind)


def init_blob(seed: int = 0) -> np.ndarray:
    """Initial parameters: weights N(0, 1/fan_in), zero biases, identity
    normalisation (replaced by data statistics before training)."""
    rng = np.random.default_rng(seed)
    blob = np.zeros(NTYPES * PER_TYPE, np.float32)
    for t in range(NTYPES):
        b = t * PER_TYPE
        off = b
        blob[off + DIN: off + 2 * DIN] = 1.0  # in_std
        off += 2 * DIN
        for fan_in, fan_out in ((DIN, HID), (HID, HID), (HID, HID), (HID, DOUT)):
            blob[off: off + fan_in * fan_out] = rng.normal(scale=math.sqrt(1.0 / fan_in), size=fan_in * fan_out)
            off += fan_in * fan_out + fan_out
        blob[off + DOUT: off + 2 * DOUT] = 1.0  # out_std
    return blob


class GuessModel:
    """A trained parameter blob on the device (``mb_guess_model``)."""

    def __init__(self, blob: np.ndarray | None = None, path: str | None = None):
        if blob is None:
            blob = np.load(path or DEFAULT_MODEL)
        blob = np.ascontiguousarray(blob, dtype=np.float32)
        if blob.size != lib().mb_guess_blob_floats():
            raise ValueError(f"parameter blob has {blob.size} floats, expected {lib().mb_guess_blob_floats()}")
        self.blob = blob
        h = ctypes.c_void_p()
        check(lib().mb_guess_model_create(blob.ctypes.data, ctypes.byref(h)))
        self.handle = h

    @staticmethod
    def available(path: str | None = None) -> bool:
        return os.path.exists(path or DEFAULT_MODEL)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            lib().mb_guess_model_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ device helpers
def _torch():
    import torch
    return torch


def _ptr(t) -> int:
    return t.data_ptr()


def _stream() -> int:
    return _torch().cuda.current_stream().cuda_stream


def atom_tables(nat):
    """0-based first orbital and orbital count per atom (s: 1, sp: 4)."""
    nor = np.where(np.asarray(nat) == 1, 1, 4).astype(np.int32)
    first = np.concatenate([[0], np.cumsum(nor)[:-1]]).astype(np.int32)
    return first, nor


class PairSet:
    """Pairs, frames and raw descriptors of one molecule on the device,
    ordered type by type (``counts`` per type)."""

    def __init__(self, nat, xyz, rpair: float = RPAIR):
        torch = _torch()
        L = lib()
        dev = torch.device("cuda")
        self.nat = torch.as_tensor(np.ascontiguousarray(nat, np.int32), device=dev)
        self.xyz = torch.as_tensor(np.ascontiguousarray(xyz, np.float64).reshape(-1, 3), device=dev)
        first, nor = atom_tables(nat)
        self.first = torch.as_tensor(first, device=dev)
        self.nor = torch.as_tensor(nor, device=dev)
        self.numat = len(nat)
        self.norbs = int(nor.sum())
        work = torch.zeros(15, dtype=torch.int32, device=dev)
        counts = (ctypes.c_int * NTYPES)()
        s = _stream()
        check(L.mb_guess_pairs_dev(self.numat, _ptr(self.nat), _ptr(self.xyz), rpair, counts, 0, None, None, None,
                                   _ptr(work), s))
        self.counts = [int(c) for c in counts]
        self.n = tot = sum(self.counts)
        self.pf = torch.empty(tot, dtype=torch.int32, device=dev)
        self.ps = torch.empty(tot, dtype=torch.int32, device=dev)
        self.pt = torch.empty(tot, dtype=torch.int32, device=dev)
        check(L.mb_guess_pairs_dev(self.numat, _ptr(self.nat), _ptr(self.xyz), rpair, counts, tot, _ptr(self.pf),
                                   _ptr(self.ps), _ptr(self.pt), _ptr(work), s))
        self.feat = torch.empty((tot, DIN), dtype=torch.float32, device=dev)
        self.frames = torch.empty((tot, 9), dtype=torch.float64, device=dev)
        self.ws = torch.empty(int(L.mb_guess_features_ws_bytes(self.numat)), dtype=torch.uint8, device=dev)
        check(L.mb_guess_features_dev(self.numat, _ptr(self.nat), _ptr(self.xyz), tot, _ptr(self.pf), _ptr(self.ps),
                                      _ptr(self.feat), _ptr(self.frames), _ptr(self.ws), s))
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)]).astype(int)

    def targets(self, p_dev_ptr: int):
        """Each pair's block of a packed device density in its frame (raw)."""
        torch = _torch()
        y = torch.empty((self.n, DOUT), dtype=torch.float32, device="cuda")
        check(lib().mb_guess_targets_dev(self.n, _ptr(self.pf), _ptr(self.ps), _ptr(self.pt), _ptr(self.frames),
                                         _ptr(self.first), _ptr(self.nor), p_dev_ptr, _ptr(y), _stream()))
        return y


# ------------------------------------------------------------------- data
@dataclass
class DataSet:
    x: list      # per type: raw descriptors (N_t x DIN, float32, device)
    y: list      # per type: raw local blocks (N_t x DOUT, float32, device)
    n_clusters: int
    seconds_scf: float
    mean_niter: float


KEEP = (1.0, 1.0, 0.3, 0.1, 0.075)   # fraction of each type's pairs kept per cluster


def generate(n_clusters: int, nmin: int = 8, nmax: int = 64, seed: int = 100, keep=KEEP,
             log_every: int = 0, kind: str = "lattice") -> DataSet:
    """Converged densities of (H2O)_n clusters, n ~ U{nmin..nmax}, from the
    plain FP64 SCF; keeps a random fraction of each type's pair blocks."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    xs = [[] for _ in range(NTYPES)]
    ys = [[] for _ in range(NTYPES)]
    t_scf, iters = 0.0, []
    for c in range(n_clusters):
        nw = int(rng.integers(nmin, nmax + 1))
        nat, xyz = make_cluster(kind, nw, int(rng.integers(1 << 30)))
        t0 = time.perf_counter()
        ctx = ScfContext(nat, xyz)
        ctx.hcore()
        r = ctx.run()
        t_scf += time.perf_counter() - t0
        iters.append(r.niter)
        ps = PairSet(nat, xyz)
        y = ps.targets(ctx.device_ptrs()["p"])
        for t in range(NTYPES):
            a, b = ps.offsets[t], ps.offsets[t + 1]
            if b == a:
                continue
            sel = torch.rand(b - a, device="cuda", generator=g) < keep[t]
            xs[t].append(ps.feat[a:b][sel])
            ys[t].append(y[a:b][sel])
        ctx.close()
        if log_every and (c + 1) % log_every == 0:
            print(f"  data: {c + 1}/{n_clusters} clusters, SCF {t_scf:.1f} s", flush=True)
    x = [torch.cat(v) if v else torch.empty((0, DIN), device="cuda") for v in xs]
    y = [torch.cat(v) if v else torch.empty((0, DOUT), device="cuda") for v in ys]
    return DataSet(x, y, n_clusters, t_scf, float(np.mean(iters)))


# ---------------------------------------------------------------- training
class Trainer:
    """Device trainer (``mb_guess_trainer``): FP32 master weights, BF16 GEMMs, Adam."""

    def __init__(self, blob: np.ndarray, max_rows: int):
        blob = np.ascontiguousarray(blob, np.float32)
        h = ctypes.c_void_p()
        check(lib().mb_guess_trainer_create(blob.ctypes.data, int(max_rows), ctypes.byref(h)))
        self.handle = h
        self.max_rows = max_rows

    @property
    def model_handle(self):
        return ctypes.c_void_p(lib().mb_guess_trainer_model(self.handle))

    def set_norm(self, t, in_mean, in_std, out_mean, out_std):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (in_mean, in_std, out_mean, out_std)]
        check(lib().mb_guess_trainer_set_norm(self.handle, t, *[a.ctypes.data for a in arrs]))

    def step(self, t: int, x, yt, lr: float, update: bool = True, want_loss: bool = False):
        loss = ctypes.c_double()
        check(lib().mb_guess_trainer_step(self.handle, t, int(x.shape[0]), _ptr(x), _ptr(yt), float(lr),
                                          int(update), ctypes.byref(loss) if want_loss else None, _stream()))
        return loss.value if want_loss else None

    def get(self):
        nf = NTYPES * PER_TYPE
        params = np.empty(nf, np.float32)
        grads = np.empty(nf, np.float32)
        check(lib().mb_guess_trainer_get(self.handle, params.ctypes.data, grads.ctypes.data))
        return params, grads

    def normalize(self, t: int, raw):
        torch = _torch()
        x = torch.empty(raw.shape, dtype=torch.int16, device="cuda")
        check(lib().mb_guess_normalize_dev(self.model_handle, t, int(raw.shape[0]), _ptr(raw), _ptr(x), _stream()))
        return x

    def norm_targets(self, t: int, yraw):
        torch = _torch()
        yt = torch.empty(yraw.shape, dtype=torch.float32, device="cuda")
        check(lib().mb_guess_norm_targets_dev(self.model_handle, t, int(yraw.shape[0]), _ptr(yraw), _ptr(yt),
                                              _stream()))
        return yt

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            lib().mb_guess_trainer_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def train(data: DataSet, epochs: int = 30, batch: int = 2048, lr: float = 2e-3, lr_min: float = 3e-5,
          seed: int = 0, log: bool = True):
    """Trains the five networks on the device; returns (blob, history)."""
    torch = _torch()
    blob = init_blob(seed)
    tr = Trainer(blob, batch)
    xs, ys = [], []
    for t in range(NTYPES):
        raw, yraw = data.x[t], data.y[t]
        if raw.shape[0] == 0:
            xs.append(None)
            ys.append(None)
            continue
        in_mean = raw.mean(0).cpu().numpy()
        in_std = raw.std(0).cpu().numpy()
        in_std = np.where(in_std > 1e-3, in_std, 1.0)
        out_mean = yraw.mean(0).cpu().numpy()
        out_std = yraw.std(0).cpu().numpy()
        out_std = np.where(out_std > 1e-6, out_std, 1.0)
        out_mean[NOUT[t]:] = 0.0
        out_std[NOUT[t]:] = 1.0
        tr.set_norm(t, in_mean, in_std, out_mean, out_std)
        xs.append(tr.normalize(t, raw))
        ys.append(tr.norm_targets(t, yraw))
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    steps_per_epoch = [0 if x is None else max(1, x.shape[0] // batch) for x in xs]
    total = epochs * sum(steps_per_epoch)
    history = []
    k = 0
    t0 = time.perf_counter()
    for ep in range(epochs):
        ep_loss = [0.0] * NTYPES
        for t in range(NTYPES):
            if xs[t] is None:
                continue
            n = xs[t].shape[0]
            perm = torch.randperm(n, device="cuda", generator=g)
            for s in range(steps_per_epoch[t]):
                idx = perm[s * batch: (s + 1) * batch]
                cur = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * k / max(1, total)))
                want = s == steps_per_epoch[t] - 1
                l = tr.step(t, xs[t][idx], ys[t][idx], cur, True, want)
                if want:
                    ep_loss[t] = l
                k += 1
        history.append(ep_loss)
        if log:
            print(f"  epoch {ep + 1}/{epochs}: loss " + " ".join(f"{v:.2e}" for v in ep_loss)
                  + f"  ({time.perf_counter() - t0:.1f} s)", flush=True)
    params, _ = tr.get()
    tr.close()
    return params, history


# -------------------------------------------------------------- evaluation
@dataclass
class EvalResult:
    n_clusters: int
    niter_std: float
    niter_learned: float
    ms_std: float           # device time of the SCF from the standard guess
    ms_learned: float       # prediction (wall, synchronised) + SCF from the learned guess
    max_dhf: float          # max |dHf| between the two converged SCFs, kcal/mol
    n_fallback: int         # SCFs from the network that did not converge (rerun from the standard guess)
    rows: list


def evaluate(model: GuessModel, n_clusters: int = 1000, nmin: int = 32, nmax: int = 128, seed: int = 777,
             log_every: int = 0, kind: str = "lattice", **run_kw) -> EvalResult:
    """Held-out (H2O)_n clusters (seeds disjoint from training): SCF from the
    standard guess and from the network, same options otherwise."""
    import torch
    rng = np.random.default_rng(seed)
    rows = []
    nfb = 0
    for c in range(n_clusters):
        nw = int(rng.integers(nmin, nmax + 1))
        nat, xyz = make_cluster(kind, nw, int(rng.integers(1 << 30)) + (1 << 30))
        ctx = ScfContext(nat, xyz)
        ctx.hcore()
        r0 = ctx.run(**run_kw)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.learned_guess(model)
        t_pred = (time.perf_counter() - t0) * 1e3
        try:
            r1 = ctx.run(guess=True, **run_kw)
            ok = r1.converged
        except Exception:
            ok = False
        if not ok:
            nfb += 1
            r1 = ctx.run(**run_kw)
        rows.append((nw, r0.niter, r1.niter, r0.t_total_ms, t_pred + r1.t_total_ms, abs(r1.escf - r0.escf)))
        ctx.close()
        if log_every and (c + 1) % log_every == 0:
            a = np.array(rows)
            print(f"  eval {c + 1}/{n_clusters}: iter {a[:, 1].mean():.2f} -> {a[:, 2].mean():.2f}, "
                  f"ms {a[:, 3].mean():.2f} -> {a[:, 4].mean():.2f}", flush=True)
    a = np.array(rows)
    return EvalResult(n_clusters, float(a[:, 1].mean()), float(a[:, 2].mean()), float(a[:, 3].mean()),
                      float(a[:, 4].mean()), float(a[:, 5].max()), nfb, rows)


def main(argv=None):
    """Generate data with the plain SCF, train, evaluate, save the blob.

    python -m mopac_gpu_b200.guess --clusters 20000 --eval 1000 --out PATH"""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--clusters", type=int, default=20000)
    ap.add_argument("--nmin", type=int, default=8)
    ap.add_argument("--nmax", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--eval", type=int, default=1000)
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--report", default=None)
    ap.add_argument("--kind", choices=["lattice", "box"], default="lattice")
    ap.add_argument("--eval-nmin", type=int, default=32)
    ap.add_argument("--eval-nmax", type=int, default=128)
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    data = generate(a.clusters, a.nmin, a.nmax, log_every=max(1, a.clusters // 10), kind=a.kind)
    t_data = time.perf_counter() - t0
    print(f"data: {a.clusters} clusters in {t_data:.1f} s (SCF {data.seconds_scf:.1f} s, mean "
          f"{data.mean_niter:.2f} iterations); rows per type {[int(x.shape[0]) for x in data.x]}", flush=True)
    t1 = time.perf_counter()
    blob, hist = train(data, epochs=a.epochs, batch=a.batch, lr=a.lr)
    t_train = time.perf_counter() - t1
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    np.save(a.out, blob)
    print(f"trained in {t_train:.1f} s -> {a.out}", flush=True)
    del data
    model = GuessModel(blob)
    ev = evaluate(model, a.eval, a.eval_nmin, a.eval_nmax, log_every=max(1, a.eval // 10), kind=a.kind)
    rep = dict(kind=a.kind, train_clusters=a.clusters, nmin=a.nmin, nmax=a.nmax, epochs=a.epochs, batch=a.batch,
               data_s=t_data, train_s=t_train, final_loss=hist[-1], eval_clusters=ev.n_clusters,
               niter_std=ev.niter_std, niter_learned=ev.niter_learned, ms_std=ev.ms_std, ms_learned=ev.ms_learned,
               max_dhf=ev.max_dhf, n_fallback=ev.n_fallback, eval_nmin=a.eval_nmin, eval_nmax=a.eval_nmax)
    print(json.dumps(rep), flush=True)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(dict(rep, rows=ev.rows), f)


if __name__ == "__main__":
    main()
