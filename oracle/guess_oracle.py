"""CPU oracle for the learned initial guess (test infrastructure only).

Only tests/, __graft_entry__.smoke() and the CPU legs of bench.py may import
this module; the product package never does.

The learned guess has no counterpart in the reference: MOPAC starts every
SCF from the diagonal guess of moldat.F90:731-760 or from a density read with
OLDENS (SCF/iter.F90:151-158).  This file is the CPU statement of the
library's own algorithm, which the CUDA kernels in csrc/guess.cu are checked
against:

  * atom pairs within ``RPAIR`` (diagonal blocks included), five pair types;
  * a local frame per pair (z along the pair axis, or towards the nearest
    neighbour for an atom's own block; x towards the nearest neighbour with a
    clear perpendicular component);
  * radial/angular descriptors of each centre's neighbours within ``RC``,
    expressed in that frame, plus each centre's long-range electrostatic
    environment (potential, field and field gradient of fixed reference
    charges on every other atom, no cutoff);
  * a 3-hidden-layer MLP (width 128, SiLU) per pair type with BF16 weights and
    activations and FP32 accumulation, forward and backward, Adam;
  * the predicted local blocks rotated back and written into the packed
    lower-triangle density.

Parity of this oracle is unpinned against the reference (the reference has no
learned guess); its pins are internal: rotation invariance of the descriptors,
exact round trips of blocks through the frames, and finite-difference
gradients.
"""
from __future__ import annotations

import numpy as np

RC = 6.0          # descriptor cutoff (Angstrom)
RPAIR = 6.0       # pairs whose blocks are predicted
NRAD = 8
RAD_MU = np.linspace(0.8, RC, NRAD)
RAD_SIG = 0.65
NANG = 10
NELEM = 2         # H, heavy
PER_CENTER = NELEM * NRAD * NANG       # 160
NPAIR_RBF = 16
PAIR_MU = np.linspace(0.8, RPAIR, NPAIR_RBF)
PAIR_SIG = 0.35
NLR = 10          # per centre: potential, field (3), field gradient (6)
# reference charges of the long-range descriptor: PM7 Mulliken charges of an
# isolated water (0.322260 / -0.644520, tests/mopac_api_test.F90:61-104)
QREF_H = 0.32226
QREF_HEAVY = -0.64452
DIN = 2 * PER_CENTER + NPAIR_RBF + 2 * NLR   # 356
HID = 128
DOUT = 16
NTYPES = 5
# pair types: 0 heavy atom's own block, 1 hydrogen's own block,
# 2 heavy-heavy, 3 heavy-hydrogen (first = heavy), 4 hydrogen-hydrogen
NOUT = np.array([10, 1, 16, 4, 1])
PERP_MIN2 = 0.01  # x reference needs |d_perp|^2 > 0.01 |d|^2
QSCALE = 1.0e5    # distance-squared ranks are floor(r^2 * QSCALE + 0.5), ties by index

# blob layout per type (float32): in_mean, in_std, W1, b1, W2, b2, W3, b3, W4,
# b4, out_mean, out_std
LAYOUT = [("in_mean", (DIN,)), ("in_std", (DIN,)), ("W1", (HID, DIN)), ("b1", (HID,)),
          ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)), ("b3", (HID,)),
          ("W4", (DOUT, HID)), ("b4", (DOUT,)), ("out_mean", (DOUT,)), ("out_std", (DOUT,))]
PER_TYPE = int(sum(np.prod(s) for _, s in LAYOUT))
TRAINABLE = ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4")


def norb(z: int) -> int:
    return 1 if z == 1 else 4


def blob_offsets():
    off, out = 0, {}
    for name, shp in LAYOUT:
        n = int(np.prod(shp))
        out[name] = (off, shp)
        off += n
    return out


def unpack_blob(blob: np.ndarray):
    offs = blob_offsets()
    types = []
    for t in range(NTYPES):
        base = t * PER_TYPE
        types.append({k: blob[base + o: base + o + int(np.prod(s))].reshape(s) for k, (o, s) in offs.items()})
    return types


def init_blob(seed: int = 0) -> np.ndarray:
    """He-style initial weights, zero biases, identity normalisation."""
    rng = np.random.default_rng(seed)
    blob = np.zeros(NTYPES * PER_TYPE, np.float32)
    for p in unpack_blob(blob):
        p["in_std"][:] = 1.0
        p["out_std"][:] = 1.0
        for w in ("W1", "W2", "W3", "W4"):
            fan_in = p[w].shape[1]
            p[w][:] = rng.normal(scale=np.sqrt(1.0 / fan_in), size=p[w].shape)
    return blob


# ------------------------------------------------------------------ BF16
def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def bf16_bits(x) -> np.ndarray:
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(h) -> np.ndarray:
    return (np.asarray(h, np.uint16).astype(np.uint32) << 16).view(np.float32)


# --------------------------------------------------------------- geometry
def _rank(r2: float, idx: int):
    return (int(np.floor(r2 * QSCALE + 0.5)), idx)


def pair_type(za: int, zb: int, same: bool) -> int:
    ha, hb = za != 1, zb != 1
    if same:
        return 0 if ha else 1
    if ha and hb:
        return 2
    if ha or hb:
        return 3
    return 4


def pair_list(nat, xyz, rpair: float = RPAIR):
    """Pairs (first, second, type) with |r| < rpair, own blocks included.

    first is the heavy atom of a heavy-hydrogen pair and the higher-numbered
    atom otherwise, so that for equal kinds the block (first, second) is the
    one the packed lower triangle stores."""
    nat = np.asarray(nat)
    xyz = np.asarray(xyz, np.float64)
    out = []
    for a in range(len(nat)):
        out.append((a, a, pair_type(nat[a], nat[a], True)))
        for b in range(a):
            d = xyz[a] - xyz[b]
            r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
            if r2 < rpair * rpair:
                t = pair_type(nat[a], nat[b], False)
                f, s = a, b
                if t == 3 and nat[a] == 1:
                    f, s = b, a
                out.append((f, s, t))
    out.sort(key=lambda q: (q[2], q[0], q[1]))
    arr = np.array(out, np.int64).reshape(-1, 3)
    return arr[:, 0], arr[:, 1], arr[:, 2]


def frame(f: int, s: int, xyz) -> np.ndarray:
    """3x3 matrix whose columns are the local x, y, z axes."""
    xyz = np.asarray(xyz, np.float64)
    n = xyz.shape[0]
    o = xyz[f]
    if f != s:
        z = xyz[s] - o
        excl = (f, s)
    else:
        best = None
        for k in range(n):
            if k == f:
                continue
            d = xyz[k] - o
            key = _rank(d[0] * d[0] + d[1] * d[1] + d[2] * d[2], k)
            if best is None or key < best[0]:
                best = (key, k)
        if best is None:
            return np.eye(3)
        z = xyz[best[1]] - o
        excl = (f, best[1])
    z = z / np.sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2])
    best = None
    for k in range(n):
        if k in excl:
            continue
        d = xyz[k] - o
        r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
        dz = d[0] * z[0] + d[1] * z[1] + d[2] * z[2]
        p2 = r2 - dz * dz
        if not p2 > PERP_MIN2 * r2:
            continue
        key = _rank(r2, k)
        if best is None or key < best[0]:
            best = (key, k, d - dz * z)
    if best is None:
        # no usable neighbour: the global axis least aligned with z
        az = np.abs(z)
        e = np.zeros(3)
        e[int(np.argmin(az))] = 1.0  # argmin takes the first on ties
        xp = e - (e @ z) * z
    else:
        xp = best[2]
    x = xp / np.sqrt(xp[0] * xp[0] + xp[1] * xp[1] + xp[2] * xp[2])
    y = np.array([z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]])
    return np.stack([x, y, z], axis=1)


def _center_features(c: int, excl, nat, xyz, R: np.ndarray) -> np.ndarray:
    out = np.zeros((NELEM, NRAD, NANG))
    o = xyz[c]
    for k in range(len(nat)):
        if k in excl:
            continue
        d = xyz[k] - o
        r2 = d @ d
        if not r2 < RC * RC:
            continue
        r = np.sqrt(r2)
        u = (d @ R) / r
        fc = 0.5 * (np.cos(np.pi * r / RC) + 1.0)
        g = np.exp(-(r - RAD_MU) ** 2 / (2.0 * RAD_SIG * RAD_SIG)) * fc
        ux, uy, uz = u
        ang = np.array([1.0, ux, uy, uz, ux * ux, uy * uy, uz * uz, ux * uy, ux * uz, uy * uz])
        out[0 if nat[k] == 1 else 1] += g[:, None] * ang[None, :]
    return out.reshape(-1)


def _center_longrange(c: int, excl, nat, xyz, R: np.ndarray) -> np.ndarray:
    """Potential, field and field gradient (xx, yy, zz, xy, xz, yz; 3 d d^T -
    r^2 I, over r^5) at centre c of reference charges on every atom not in
    excl, in the frame R."""
    out = np.zeros(NLR)
    o = xyz[c]
    for k in range(len(nat)):
        if k in excl:
            continue
        q = QREF_H if nat[k] == 1 else QREF_HEAVY
        d = (xyz[k] - o) @ R
        r2 = d @ d
        r = np.sqrt(r2)
        r3 = r2 * r
        r5 = r3 * r2
        x, y, z = d
        out += q * np.array([1.0 / r, x / r3, y / r3, z / r3, (3 * x * x - r2) / r5, (3 * y * y - r2) / r5,
                             (3 * z * z - r2) / r5, 3 * x * y / r5, 3 * x * z / r5, 3 * y * z / r5])
    return out


def features(nat, xyz, F, S, T):
    """Raw descriptors (npairs x DIN, float64) and frames (npairs x 3 x 3)."""
    nat = np.asarray(nat)
    xyz = np.asarray(xyz, np.float64)
    X = np.zeros((len(F), DIN))
    Rs = np.zeros((len(F), 3, 3))
    for q, (f, s) in enumerate(zip(F, S)):
        R = frame(int(f), int(s), xyz)
        Rs[q] = R
        lr0 = 2 * PER_CENTER + NPAIR_RBF
        if f == s:
            X[q, :PER_CENTER] = _center_features(int(f), (int(f),), nat, xyz, R)
            X[q, lr0:lr0 + NLR] = _center_longrange(int(f), (int(f),), nat, xyz, R)
        else:
            ex = (int(f), int(s))
            X[q, :PER_CENTER] = _center_features(int(f), ex, nat, xyz, R)
            X[q, PER_CENTER:2 * PER_CENTER] = _center_features(int(s), ex, nat, xyz, R)
            d = xyz[s] - xyz[f]
            r = np.sqrt(d @ d)
            X[q, 2 * PER_CENTER:lr0] = np.exp(-(r - PAIR_MU) ** 2 / (2.0 * PAIR_SIG * PAIR_SIG))
            X[q, lr0:lr0 + NLR] = _center_longrange(int(f), ex, nat, xyz, R)
            X[q, lr0 + NLR:] = _center_longrange(int(s), ex, nat, xyz, R)
    return X, Rs


def _umat(z: int, R: np.ndarray) -> np.ndarray:
    if z == 1:
        return np.ones((1, 1))
    u = np.zeros((4, 4))
    u[0, 0] = 1.0
    u[1:, 1:] = R   # MOPAC's sp order: s, px, py, pz
    return u


TRI4 = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2), (3, 0), (3, 1), (3, 2), (3, 3)]


def first_orbitals(nat):
    nf = np.zeros(len(nat) + 1, np.int64)
    for a, z in enumerate(nat):
        nf[a + 1] = nf[a] + norb(int(z))
    return nf


def local_blocks(p_packed, nat, F, S, T, Rs) -> np.ndarray:
    """Training targets: each pair's block of P in its local frame (npairs x DOUT)."""
    nat = np.asarray(nat)
    nf = first_orbitals(nat)
    n = int(nf[-1])
    from oracle.scf_oracle import unpack
    P = unpack(np.asarray(p_packed), n)
    Y = np.zeros((len(F), DOUT))
    for q, (f, s, t) in enumerate(zip(F, S, T)):
        B = P[nf[f]:nf[f + 1], nf[s]:nf[s + 1]]
        L = _umat(nat[f], Rs[q]).T @ B @ _umat(nat[s], Rs[q])
        if t == 0:
            Y[q, :10] = [L[i, j] for i, j in TRI4]
        else:
            Y[q, :L.size] = L.reshape(-1)
    return Y


def assemble(nat, F, S, T, Rs, Y) -> np.ndarray:
    """Packed lower-triangle density from local blocks (pairs not listed stay 0)."""
    nat = np.asarray(nat)
    nf = first_orbitals(nat)
    n = int(nf[-1])
    P = np.zeros((n, n))
    for q, (f, s, t) in enumerate(zip(F, S, T)):
        nr, nc = norb(int(nat[f])), norb(int(nat[s]))
        if t == 0:
            L = np.zeros((4, 4))
            for v, (i, j) in zip(Y[q, :10], TRI4):
                L[i, j] = L[j, i] = v
        else:
            L = np.asarray(Y[q, :nr * nc], np.float64).reshape(nr, nc)
        B = _umat(nat[f], Rs[q]) @ L @ _umat(nat[s], Rs[q]).T
        P[nf[f]:nf[f + 1], nf[s]:nf[s + 1]] = B
        P[nf[s]:nf[s + 1], nf[f]:nf[f + 1]] = B.T
    from oracle.scf_oracle import pack
    return pack(P)


# -------------------------------------------------------------------- MLP
def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    sg = 1.0 / (1.0 + np.exp(-z))
    return sg * (1.0 + z * (1.0 - sg))


def normalize(p, X) -> np.ndarray:
    """Raw descriptors -> BF16 network input."""
    return bf16((np.asarray(X, np.float32) - p["in_mean"]) / p["in_std"])


def forward(p, x, exact: bool = False):
    """x: BF16-valued float32 (n x DIN).  Returns (y, cache).

    exact=True drops every BF16/FP32 rounding (float64 throughout): the
    mathematical function, for finite-difference checks."""
    rnd = (lambda v: np.asarray(v, np.float64)) if exact else bf16
    f32 = (lambda v: np.asarray(v, np.float64)) if exact else (lambda v: np.asarray(v, np.float32))
    W = [rnd(p[k]) for k in ("W1", "W2", "W3", "W4")]
    b = [np.asarray(p[k], np.float64) if exact else p[k] for k in ("b1", "b2", "b3", "b4")]
    acts, zs = [f32(x)], []
    a = acts[0]
    for layer in range(3):
        z = f32(a.astype(np.float64) @ W[layer].T.astype(np.float64)) + b[layer]
        zs.append(z)
        a = rnd(f32(silu(z.astype(np.float64))))
        acts.append(a)
    y = f32(a.astype(np.float64) @ W[3].T.astype(np.float64)) + b[3]
    return y, (acts, zs, W)


def loss_and_grads(p, x, yt, nout: int, exact: bool = False):
    """Mean squared error over the type's valid output slots and its gradients.

    yt: normalised targets (n x DOUT).  The backward pass follows the kernels:
    every GEMM operand is BF16, every product accumulates in FP32 (exact=True:
    float64 without rounding)."""
    rnd = (lambda v: np.asarray(v, np.float64)) if exact else bf16
    f32 = (lambda v: np.asarray(v, np.float64)) if exact else (lambda v: np.asarray(v, np.float32))
    n = x.shape[0]
    y, (acts, zs, W) = forward(p, x, exact)
    mask = np.zeros(DOUT)
    mask[:nout] = 1.0
    r = (np.asarray(y, np.float64) - yt) * mask
    loss = float((r ** 2).sum() / (n * nout))
    dz = rnd(f32((2.0 / (n * nout)) * r))
    g = {}
    for layer in (3, 2, 1, 0):
        a_prev = acts[layer]
        g[f"W{layer + 1}"] = f32(dz.astype(np.float64).T @ a_prev.astype(np.float64))
        g[f"b{layer + 1}"] = f32(dz.astype(np.float64).sum(axis=0))
        if layer > 0:
            da = f32(dz.astype(np.float64) @ W[layer].astype(np.float64))
            dz = rnd(f32(da * dsilu(zs[layer - 1].astype(np.float64))))
    return loss, g, y


def adam(p, g, m, v, step: int, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
    """One Adam step on the trainable arrays (in place)."""
    c1 = 1.0 - b1 ** step
    c2 = 1.0 - b2 ** step
    for k in TRAINABLE:
        m[k][:] = b1 * m[k] + (1 - b1) * g[k]
        v[k][:] = b2 * v[k] + (1 - b2) * g[k] * g[k]
        p[k][:] = p[k] - lr * (m[k] / c1) / (np.sqrt(v[k] / c2) + eps)


def purify(p_packed, n: int, steps: int = 1) -> np.ndarray:
    """McWeeny purification of a packed total density: D = P/2,
    D <- 3 D^2 - 2 D^3 (steps times), P = 2 D (symmetric part)."""
    from oracle.scf_oracle import pack, unpack
    D = unpack(np.asarray(p_packed, np.float64), n) * 0.5
    for _ in range(steps):
        D2 = D @ D
        D = 3.0 * D2 - 2.0 * (D2 @ D)
    return pack(D + D.T)


def predict_density(blob, nat, xyz) -> np.ndarray:
    """The learned guess end to end on the CPU (packed total density)."""
    types = unpack_blob(blob)
    F, S, T = pair_list(nat, xyz)
    X, Rs = features(nat, xyz, F, S, T)
    Y = np.zeros((len(F), DOUT))
    for t in range(NTYPES):
        sel = T == t
        if not sel.any():
            continue
        p = types[t]
        y, _ = forward(p, normalize(p, X[sel]))
        Y[sel] = y.astype(np.float64) * p["out_std"] + p["out_mean"]
    return assemble(nat, F, S, T, Rs, Y)
