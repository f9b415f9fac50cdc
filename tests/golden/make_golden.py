"""Generates the golden fixtures tests/golden/*.npz from the oracle.

The oracle's layout and tables are pinned to the reference's own code
(oracle/_ref, tests/test_oracle_pin.py) and its classification / traversal /
geometry to the reference's generated GLSL run as C++ (tests/test_glsl_pin.py);
the fixtures freeze its output on small seeded inputs so that every machine
(including ones without the HPMC tree) checks against the same numbers.

Inputs are regenerated from the seeds in CASES; only outputs are stored.
Run from the repository root:  python -m tests.golden.make_golden
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def make_field(kind: str, shape, seed: int):
    rng = np.random.default_rng(seed)
    fz, fy, fx = shape
    if kind == "metaballs":
        from hpmc_b200 import datasets

        c = rng.uniform(0.2, 0.8, size=(6, 3))
        r = rng.uniform(0.05, 0.2, size=6)
        return datasets.metaballs(0, c, r, shape=(fx, fy, fz))
    if kind == "ties_u8":
        return rng.integers(120, 137, size=shape).astype(np.uint8)
    if kind == "normal":
        return rng.normal(size=shape).astype(np.float32)
    raise ValueError(kind)


CASES = {
    "metaballs_16": dict(kind="metaballs", shape=(16, 16, 16), seed=0, iso=1.0),
    "metaballs_odd": dict(kind="metaballs", shape=(13, 21, 17), seed=1, iso=0.8, extent=(2.0, 1.0, 0.5)),
    "ties_u8": dict(kind="ties_u8", shape=(10, 12, 9), seed=2, iso=128.0),
    "ties_unorm8": dict(kind="ties_u8", shape=(9, 8, 11), seed=3, iso=128.0 / 255.0, unorm=True),
    "normal_grid": dict(kind="normal", shape=(11, 10, 12), seed=4, iso=0.0, cells=(9, 8, 7)),
    "binary": dict(kind="normal", shape=(8, 9, 10), seed=5, iso=0.0, binary=True),
    "tiny": dict(kind="normal", shape=(3, 3, 3), seed=6, iso=0.0),
}


def run_case(O, kind, shape, seed, iso, extent=(1.0, 1.0, 1.0), cells=None, binary=False, unorm=False):
    field = make_field(kind, shape, seed)
    fz, fy, fx = shape
    L = O.layout((fx, fy, fz), cells)
    codes = O.codes(field, L, iso, binary=binary, unorm=unorm)
    levels, total = O.pyramid(codes, L)
    out = {"codes": codes, "total": np.array([total], np.uint64),
           "layout": np.array(L.tile + L.layout + (L.size_l2, L.size), np.int32)}
    for j, lv in enumerate(levels):
        out[f"level{j}"] = lv
    out["level0_texture"] = O.level0_texture(codes, L)
    cell, code, k, edge = O.traverse(codes, levels, L, 0, total)
    out.update(cell=cell, code=code, k=k, edge=edge)
    for name, mode in (("fwd", O.NORMALS_FORWARD), ("ctr", O.NORMALS_CENTRAL)):
        t, pos, nrm = O.geometry(field, L, iso, cell, code, k, edge, binary=binary, normal_mode=mode,
                                 extent=extent, unorm=unorm)
        out[f"t_{name}"] = t
        out[f"pos_{name}"] = pos
        out[f"nrm_{name}"] = nrm
    return out


def main():
    from oracle import oracle as O

    for name, case in CASES.items():
        out = run_case(O, **case)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, int(out["total"][0]), "vertices")


if __name__ == "__main__":
    main()
