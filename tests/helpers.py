"""Shared fixtures for the parity tests: systems, oracle integrals, GPU tensors."""
from __future__ import annotations

import json
import os

import numpy as np

from oracle import scf_oracle as so

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_values.json")))


def small_systems():
    from mopac_gpu_b200 import workloads as wl
    out = {}
    for k in ("co2_1scf", "propane", "h2o_api"):
        out[k] = (np.array(GOLDEN[k]["nat"], np.int32), np.array(GOLDEN[k]["xyz"], float))
    out["water16"] = wl.water_lattice(16)
    rng = np.random.default_rng(5)
    out["heptane"] = wl.alkane(7, rng)
    return out


def oracle_system(nat, xyz):
    return so.make_system(nat, xyz)


def mixed_density(s, seed=0):
    """A symmetric packed density with realistic magnitudes (oracle SCF after
    two iterations plus noise), so every Fock branch sees nonzero data."""
    rng = np.random.default_rng(seed)
    r = so.iter_scf(s, itrmax=2)
    p = r.p.copy()
    p += rng.normal(scale=1e-3, size=p.shape)
    return p
