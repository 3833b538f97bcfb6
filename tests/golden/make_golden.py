"""Generate the golden fixtures from the reference itself.

Runs the reference's own CPU path (oracle/_ref/mdgpu_ref_harness, compiled from
the reference sources by ``make -C oracle ref``) on seeded synthetic matrices
and stores what it produced:

* small cases: the full arrays (permutation, elimination tree, postorder,
  column counts, supernode partition and children, L pattern and values,
  solution) in ``<case>.npz``;
* larger cases: SHA-256 digests of the same arrays (little-endian bytes) in
  ``manifest.json``, so the fixtures stay small while still pinning every bit.

Only this script reads the reference; the tests read the committed fixtures.
Usage:  python tests/golden/make_golden.py   (takes about a minute)
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mdgpu_b200 import matgen as mg  # noqa: E402
from oracle import oracle as O  # noqa: E402

INT_KEYS = ["perm", "parent", "post", "count0", "count", "rn_perm", "sn_nodo", "sn_cols",
            "sn_childptr", "sn_child", "Lp", "Ap", "Ai", "Li"]
F64_KEYS = ["Ax", "Lx", "b", "x"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# (case name, generator spec, flags, store full arrays?, run the factor?)
CASES = [
    ("cfg1_2d100_amd_sn", ("2d", 100), dict(amd=True, mode="sn"), True, True),
    ("2d100_amd_nodal", ("2d", 100), dict(amd=True, mode="nodal"), False, True),
    ("2d100_nat_sn", ("2d", 100), dict(amd=False, mode="sn"), False, True),
    ("2d100_amd_rn4", ("2d", 100), dict(amd=True, mode="rn", rn_zeros=4), False, True),
    ("2d100_amd_rn16", ("2d", 100), dict(amd=True, mode="rn", rn_zeros=16), False, True),
    ("3d10_amd_sn", ("3d", 10, 0, 1.0, 1e-3), dict(amd=True, mode="sn"), True, True),
    ("3d16_amd_sn", ("3d", 16, 0, 1.0, 1e-3), dict(amd=True, mode="sn"), False, True),
    ("3d16_amd_sn_b8", ("3d", 16, 0, 1.0, 1e-3), dict(amd=True, mode="sn", block=8), False, True),
    ("3d16_amd_nodal", ("3d", 16, 0, 1.0, 1e-3), dict(amd=True, mode="nodal"), False, True),
    ("3d16_nat_sn", ("3d", 16, 0, 1.0, 1e-3), dict(amd=False, mode="sn"), False, True),
    ("3d16_amd_rn4", ("3d", 16, 0, 1.0, 1e-3), dict(amd=True, mode="rn", rn_zeros=4), False, True),
    ("3d16_amd_rn16", ("3d", 16, 0, 1.0, 1e-3), dict(amd=True, mode="rn", rn_zeros=16), False,
     True),
    ("rnd300_amd_sn", ("rnd", 300, 0.02, 1), dict(amd=True, mode="sn"), True, True),
    ("rnd300_nat_nodal", ("rnd", 300, 0.02, 1), dict(amd=False, mode="nodal"), True, True),
    ("rnd300_amd_rn8", ("rnd", 300, 0.02, 1), dict(amd=True, mode="rn", rn_zeros=8), True, True),
    ("3d32_amd_sn", ("3d", 32, 0, 1.0, 1e-3), dict(amd=True, mode="sn"), False, True),
    ("3d48_amd_sn_sym", ("3d", 48, 0, 1.0, 1e-2), dict(amd=True, mode="sn"), False, False),
    ("cfg2_3d64_amd_sn_sym", ("3d", 64, 0, 1.0, 1e-3), dict(amd=True, mode="sn"), False, False),
]


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


def main():
    if not os.path.exists(O.REF_HARNESS):
        sys.exit("build the reference first: make -C oracle ref")
    manifest = {}
    tmp = tempfile.mkdtemp(prefix="mdgpu_golden_")
    try:
        for name, spec, flags, full, factor in CASES:
            n, Ap, Ai, Ax = make_matrix(spec)
            mfile = os.path.join(tmp, name + ".txt")
            mg.write_triplets(mfile, n, Ap, Ai, Ax)
            bfile = os.path.join(tmp, name + ".b")
            b = mg.rhs_uniform(n, seed=0)
            b.tofile(bfile)
            flags = dict(flags)
            block = flags.pop("block", 0)
            R = O.run_reference(mfile, os.path.join(tmp, name), block=block, bfile=bfile,
                                factor=factor, **flags)
            entry = {"spec": list(spec), "flags": dict(flags, block=block), "factor": factor,
                     "meta": R["meta"],
                     "input_sha": {"Ap": digest(Ap), "Ai": digest(Ai), "Ax": digest(Ax)},
                     "sha": {}}
            arrays = {}
            for k in INT_KEYS + F64_KEYS:
                if k not in R:
                    continue
                entry["sha"][k] = digest(R[k])
                if full:
                    arrays[k] = R[k]
            if full:
                np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
            manifest[name] = entry
            print(name, R["meta"])
    finally:
        shutil.rmtree(tmp)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
