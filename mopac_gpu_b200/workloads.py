"""Seeded synthetic geometries for the benchmark workloads.

No public data set is involved; every system is generated here from a seed.
  water_lattice(16)   (H2O)_16: O on a 4x4x1 lattice, 2.9 A spacing, +-0.2 A
                      uniform jitter, rigid waters (O-H 0.96 A, H-O-H 104.5
                      deg) with uniform random orientations.
  water_box(512)      (H2O)_512 at 1.0 g/cm^3 (cubic cell ~24.8 A, no
                      periodicity) by random sequential insertion with
                      O-O >= 2.6 A; insertions that put any intermolecular
                      atom pair closer than 1.4 A are also rejected.
  alkane(n)           C_nH_(2n+2): C-C 1.54 A, C-H 1.09 A, tetrahedral angles,
                      C-C-C-C torsions from {60, 180, 300} deg +- U(10) deg;
                      a conformer whose non-bonded atoms clash (H...H < 1.7,
                      C...H < 2.0, C...C < 2.45 A beyond geminal pairs) is
                      redrawn.
  alkane_batch(4096)  n ~ U{3..20}.
Atomic numbers: H 1, C 6, O 8.  Coordinates in Angstrom.
"""
from __future__ import annotations

import numpy as np

OH = 0.96
HOH = np.deg2rad(104.5)
TETRA = np.arccos(-1.0 / 3.0)  # 109.47 deg
WATER_MASS_G = 18.01528 / 6.02214076e23


def _rand_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def _water_frame() -> np.ndarray:
    h = HOH / 2
    return np.array([[0.0, 0.0, 0.0],
                     [OH * np.sin(h), OH * np.cos(h), 0.0],
                     [-OH * np.sin(h), OH * np.cos(h), 0.0]])


def _place_water(o: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    return o + _water_frame() @ _rand_rotation(rng).T


def water_lattice(n: int = 16, seed: int = 1234, spacing: float = 2.9, jitter: float = 0.2, nx: int | None = None):
    """(H2O)_n on an nx x ny x nz lattice (default 4x4x1 for n = 16)."""
    rng = np.random.default_rng(seed)
    if nx is None:
        if n == 16:
            dims = (4, 4, 1)
        else:
            s = int(np.ceil(n ** (1.0 / 3.0)))
            dims = (s, s, s)
    else:
        dims = (nx, int(np.ceil(n / nx)), 1)
    pts = []
    for k in range(dims[2]):
        for j in range(dims[1]):
            for i in range(dims[0]):
                if len(pts) < n:
                    pts.append(np.array([i, j, k], float) * spacing)
    nat, xyz = [], []
    for p in pts:
        o = p + rng.uniform(-jitter, jitter, size=3)
        w = _place_water(o, rng)
        nat += [8, 1, 1]
        xyz.append(w)
    return np.array(nat, np.int32), np.concatenate(xyz)


def water_box(n: int = 512, seed: int = 2024, density_g_cm3: float = 1.0, min_oo: float = 2.6,
              min_other: float = 1.4, max_tries: int = 2_000_000):
    """(H2O)_n by random sequential insertion in a cube at the given density."""
    rng = np.random.default_rng(seed)
    vol = n * WATER_MASS_G / density_g_cm3 * 1e24  # A^3
    edge = vol ** (1.0 / 3.0)
    cell = 3.0
    ncell = max(1, int(edge // cell))
    grid: dict = {}
    waters = []

    def cidx(p):
        return tuple(np.minimum((p / edge * ncell).astype(int), ncell - 1))

    tries = 0
    while len(waters) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("random sequential insertion did not converge")
        o = rng.uniform(0.0, edge, size=3)
        w = _place_water(o, rng)
        c = cidx(o)
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in grid.get((c[0] + dx, c[1] + dy, c[2] + dz), ()):
                        other = waters[q]
                        if np.sum((other[0] - w[0]) ** 2) < min_oo * min_oo:
                            ok = False
                            break
                        d = other[:, None, :] - w[None, :, :]
                        dd = np.einsum("ijk,ijk->ij", d, d)
                        dd[0, 0] = 1e9
                        if dd.min() < min_other * min_other:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            grid.setdefault(c, []).append(len(waters))
            waters.append(w)
    nat = np.array([8, 1, 1] * n, np.int32)
    return nat, np.concatenate(waters), edge


def _zmat_place(a, b, c, bond, angle, dihedral):
    """Position of a new atom d with |d-c| = bond, angle(b,c,d), dihedral(a,b,c,d)."""
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    n /= np.linalg.norm(n)
    m = np.cross(n, bc)
    d2 = np.array([-bond * np.cos(angle), bond * np.sin(angle) * np.cos(dihedral), bond * np.sin(angle) * np.sin(dihedral)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def _clash(nat: np.ndarray, xyz: np.ndarray) -> bool:
    d = np.linalg.norm(xyz[:, None, :] - xyz[None, :, :], axis=-1)
    n = len(nat)
    lim = np.where((nat[:, None] == 1) & (nat[None, :] == 1), 1.7,
                   np.where((nat[:, None] == 6) & (nat[None, :] == 6), 2.45, 2.0))
    # bonded and geminal (1-3) pairs are exempt: distance below 2.6 A between
    # atoms that share a neighbour is expected; mark them by chain topology
    iu = np.triu_indices(n, 1)
    bad = d[iu] < lim[iu]
    if not bad.any():
        return False
    # exempt pairs within two bonds: C-C 1.54/2.52, C-H 1.09/2.17, H-H(gem) 1.78
    for i, j in zip(iu[0][bad], iu[1][bad]):
        if nat[i] == 6 and nat[j] == 6 and d[i, j] > 1.4 and d[i, j] < 1.6:
            continue
        if nat[i] != nat[j] and d[i, j] < 1.2:
            continue
        if nat[i] == 6 and nat[j] == 6 and abs(d[i, j] - 2.515) < 0.05:
            continue
        if nat[i] != nat[j] and abs(d[i, j] - 2.17) < 0.06:
            continue
        if nat[i] == 1 and nat[j] == 1 and abs(d[i, j] - 1.78) < 0.03:
            continue
        return True
    return False


def alkane(nc: int, rng: np.random.Generator, max_tries: int = 1000):
    """Linear alkane C_nH_(2n+2) with random staggered torsions, clash-free."""
    for _ in range(max_tries):
        nat, xyz = _alkane_once(nc, rng)
        if not _clash(nat, xyz):
            return nat, xyz
    raise RuntimeError("no clash-free conformer found")


def _alkane_once(nc: int, rng: np.random.Generator):
    cc, ch = 1.54, 1.09
    carbons = [np.zeros(3), np.array([cc, 0.0, 0.0])]
    if nc >= 3:
        carbons.append(carbons[1] + cc * np.array([-np.cos(TETRA), np.sin(TETRA), 0.0]))
    prev = 180.0
    for i in range(3, nc):
        # trans or gauche, never a gauche+ gauche- pair (the syn-pentane clash)
        choices = [180.0, prev] if prev != 180.0 else [60.0, 180.0, 300.0]
        t = float(rng.choice(choices))
        prev = t
        tor = np.deg2rad(t + rng.uniform(-10.0, 10.0))
        carbons.append(_zmat_place(carbons[i - 3], carbons[i - 2], carbons[i - 1], cc, TETRA, tor))
    carbons = carbons[:nc]
    hs = []
    for i, c in enumerate(carbons):
        nbr = [carbons[j] for j in (i - 1, i + 1) if 0 <= j < nc]
        if len(nbr) == 2:
            u1 = (c - nbr[0]) / np.linalg.norm(c - nbr[0])
            u2 = (c - nbr[1]) / np.linalg.norm(c - nbr[1])
            bis = u1 + u2
            bis /= np.linalg.norm(bis)
            perp = np.cross(u1, u2)
            perp /= np.linalg.norm(perp)
            half = TETRA / 2
            for s in (1.0, -1.0):
                hs.append(c + ch * (np.cos(half) * bis + s * np.sin(half) * perp))
        else:
            # terminal carbon: three H staggered about the C-C axis
            a = nbr[0]
            ref = carbons[i + 2] if i == 0 and nc > 2 else (carbons[i - 2] if nc > 2 else a + np.array([0.0, 1.0, 0.3]))
            for k in range(3):
                hs.append(_zmat_place(ref, a, c, ch, TETRA, np.deg2rad(180.0 + 120.0 * k)))
    nat = np.array([6] * nc + [1] * len(hs), np.int32)
    return nat, np.vstack([np.array(carbons), np.array(hs)])


def alkane_batch(count: int = 4096, seed: int = 77, nmin: int = 3, nmax: int = 20):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nc = int(rng.integers(nmin, nmax + 1))
        out.append(alkane(nc, rng))
    return out


def formula(nat) -> str:
    from collections import Counter
    c = Counter(int(z) for z in nat)
    sym = {1: "H", 6: "C", 8: "O"}
    return "".join(f"{sym[z]}{c[z]}" for z in (6, 1, 8) if c[z])


def mozyme_lmos(nat, xyz, radius: float = 4.0, seed: int = 11, per_heavy: int = 4, pad_atoms: int = 0):
    """Synthetic occupied LMOs in the reference's MOZYME_C arrays, for kernel
    tests and timing: every O or C atom owns `per_heavy` LMOs that cover the
    atom itself, then every other atom within `radius` Angstrom in order of
    distance (the way diagg2 grows an LMO outward); coefficients decay with
    distance.  pad_atoms empty atom slots (and 4 coefficients each) follow
    every LMO, the room diagg2 may grow it into.  Returns (iorbs, (ncf, nncf,
    icocc, ncocc, cocc)) with icocc 1-based and nncf/ncocc 0-based starts."""
    nat = np.asarray(nat)
    xyz = np.asarray(xyz, float).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    iorbs = np.where(nat == 1, 1, 4).astype(np.int32)
    ncf, nncf, icocc, ncocc, cocc = [], [], [], [], []
    heavy = np.nonzero(nat != 1)[0]
    for a in heavy:
        d = np.linalg.norm(xyz - xyz[a], axis=1)
        near = np.nonzero(d < radius)[0]
        near = near[np.argsort(d[near], kind="stable")]
        for _ in range(per_heavy):
            nncf.append(len(icocc))
            ncocc.append(len(cocc))
            ncf.append(len(near))
            vec = []
            for b in near:
                icocc.append(int(b) + 1)
                vec.extend((rng.normal(size=iorbs[b]) * np.exp(-d[b] / 1.5)).tolist())
            vec = np.asarray(vec)
            cocc.extend((vec / np.linalg.norm(vec)).tolist())  # unit LMOs
            icocc.extend([0] * pad_atoms)
            cocc.extend([0.0] * (4 * pad_atoms))
    lmos = (np.array(ncf, np.int32), np.array(nncf, np.int32), np.array(icocc, np.int32),
            np.array(ncocc, np.int32), np.array(cocc, np.float64))
    return iorbs, lmos
