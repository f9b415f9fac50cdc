"""The oracle against the reference's own generated GLSL, run on the CPU
(oracle/glsl_pin.py compiles the shader text the reference's generator emits
against a small GLSL-subset runtime).

Pinned bit-exactly: the base level texture (counts + code fractions, masked
cells, padding texels), every reduction level, and the vertex count; per
vertex, the positions and normals of the FP32 shader arithmetic agree with the
oracle's FP64 geometry to FP32 rounding -- which also pins the vertex order.
Texture-field mode with forward-difference normals (the reference's
non-gradient path, shadergen.cpp:436-565).
"""
from __future__ import annotations

import numpy as np
import pytest

pytest.importorskip("oracle.glsl_pin")


def _glsl():
    from oracle import glsl_pin

    return glsl_pin


CASES = [
    ((8, 9, 10), None, (1.0, 1.0, 1.0), 0),
    ((17, 12, 9), None, (2.0, 1.0, 0.5), 1),
    ((33, 20, 7), (20, 15, 5), (1.0, 1.0, 1.0), 2),   # grid smaller than the lattice
    ((5, 40, 12), None, (1.0, 3.0, 1.0), 3),
]


@pytest.mark.parametrize("lattice,cells,extent,seed", CASES)
def test_oracle_matches_reference_glsl(oracle, lattice, cells, extent, seed):
    rng = np.random.default_rng(seed)
    fx, fy, fz = lattice
    field = rng.normal(size=(fz, fy, fx)).astype(np.float32)
    field[rng.random(field.shape) < 0.05] = 0.0  # samples equal to iso (ties)
    iso = 0.0
    levels_g, n_g, pos_g, nrm_g = _glsl().run(field, iso, cells=cells, extent=extent)

    L = oracle.layout(lattice, cells)
    codes = oracle.codes(field, L, iso)
    tex = oracle.level0_texture(codes, L)
    assert np.array_equal(levels_g[0], tex), "base level texture differs"
    levels, total = oracle.pyramid(codes, L)
    for m in range(1, L.size_l2 + 1):
        w = L.size >> m
        got = levels_g[m]
        # mip m texel (i, j) channel c <-> oracle level m entry 4*morton(i, j) + c
        idx = np.zeros((w, w), np.int64)
        for j in range(w):
            for i in range(w):
                mi = 0
                for b in range(16):
                    mi |= ((i >> b) & 1) << (2 * b) | ((j >> b) & 1) << (2 * b + 1)
                idx[j, i] = mi
        expect = levels[m][(4 * idx[..., None] + np.arange(4)).reshape(-1)].reshape(w, w, 4)
        assert np.array_equal(got.astype(np.int64), expect.astype(np.int64)), f"mip level {m} differs"
    assert n_g == total
    cell, code, k, edge = oracle.traverse(codes, levels, L, 0, total)
    _, pos, nrm = oracle.geometry(field, L, iso, cell, code, k, edge, normal_mode=0, extent=extent)
    spacing = np.array(extent) / np.array(L.cells)
    dp = np.abs(pos_g.astype(np.float64) - pos)
    assert (dp <= 4e-6 * (np.abs(pos) + spacing)).all(), float(dp.max())
    scale = np.abs(nrm).max(1, keepdims=True) + 1e-30
    assert (np.abs(nrm_g.astype(np.float64) - nrm) <= 1e-5 * scale).all()


def test_oracle_matches_reference_glsl_unorm8(oracle):
    """A GL_ALPHA / GL_UNSIGNED_BYTE volume (apps/texture3d) reads as b/255:
    the shaders see those floats; the oracle classifies the bytes (UNORM8)."""
    rng = np.random.default_rng(11)
    vol = rng.integers(100, 156, size=(9, 12, 14)).astype(np.uint8)
    iso = np.float32(128) / np.float32(255)  # samples equal to iso: ties
    levels_g, n_g, pos_g, nrm_g = _glsl().run((vol.astype(np.float32) / np.float32(255)), float(iso))
    L = oracle.layout((14, 12, 9))
    codes = oracle.codes(vol, L, float(iso), unorm=True)
    assert np.array_equal(levels_g[0], oracle.level0_texture(codes, L))
    _, total = oracle.pyramid(codes, L)
    assert n_g == total > 0
