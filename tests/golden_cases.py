"""Helpers that rebuild the golden cases' inputs and compare against digests."""
import hashlib
import json
import os

import numpy as np

from mdgpu_b200 import matgen as mg

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def manifest():
    with open(os.path.join(HERE, "manifest.json")) as f:
        return json.load(f)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make_matrix(spec):
    kind = spec[0]
    if kind == "2d":
        return mg.laplacian_2d_5pt(spec[1])
    if kind == "3d":
        _, side, seed, sigma, shift = spec
        return mg.laplacian_3d_varcoef(side, seed=seed, sigma=sigma, shift=shift)
    if kind == "rnd":
        _, n, dens, seed = spec
        return mg.random_spd(n, dens, seed=seed)
    raise ValueError(spec)


def load_full(name):
    p = os.path.join(HERE, name + ".npz")
    if not os.path.exists(p):
        return None
    with np.load(p) as z:
        return {k: z[k] for k in z.files}
