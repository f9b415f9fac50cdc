"""The oracle against the reference's own generated GLSL, run on the CPU
(oracle/glsl_pin.py compiles the shader text the reference's generator emits
against a small GLSL-subset runtime).

Pinned bit-exactly: the base level texture (counts + code fractions, masked
cells, padding texels), every reduction level, and the vertex count; per
vertex, the positions and normals of the FP32 shader arithmetic agree with the
oracle's FP64 geometry to FP32 rounding -- which also pins the vertex order.
Modes: texture fields with forward-difference normals (shadergen.cpp:436-565),
binary fields (midpoints and table normals, shadergen.cpp:99-101, 507-522),
RGBA gradient textures (shadergen.cpp:260-266, 539-551), and the custom-fetch
path with the Cayley demo's own GLSL snippet (apps/cayley/cayley.cpp:75-94,
shadergen.cpp:270-286), gradient off and on; the 64^3 metaballs workload at
its full size.
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


def _morton_index(w):
    """mip texel (i, j) -> its Morton index (i on the even bits)."""
    i = np.arange(w, dtype=np.int64)
    spread = np.zeros(w, np.int64)
    for b in range(16):
        spread |= ((i >> b) & 1) << (2 * b)
    return spread[None, :] | (spread[:, None] << 1)


def _check_levels(levels_g, codes, L, oracle):
    """Base texture and every mip level bit-exact; returns the oracle's levels and count."""
    assert np.array_equal(levels_g[0], oracle.level0_texture(codes, L)), "base level texture differs"
    levels, total = oracle.pyramid(codes, L)
    for m in range(1, L.size_l2 + 1):
        w = L.size >> m
        # mip m texel (i, j) channel c <-> oracle level m entry 4*morton(i, j) + c
        idx = _morton_index(w)
        expect = levels[m][(4 * idx[..., None] + np.arange(4)).reshape(-1)].reshape(w, w, 4)
        assert np.array_equal(levels_g[m].astype(np.int64), expect.astype(np.int64)), f"mip level {m} differs"
    return levels, total


def _check_geometry(pos_g, nrm_g, pos, nrm, L, extent, pos_tol=4e-6, nrm_tol=1e-5, spacing_tol=0.0):
    spacing = np.array(extent) / np.array(L.cells)
    dp = np.abs(pos_g.astype(np.float64) - pos)
    assert (dp <= pos_tol * (np.abs(pos) + spacing) + spacing_tol * spacing).all(), float(dp.max())
    scale = np.abs(nrm).max(1, keepdims=True) + 1e-30
    assert (np.abs(nrm_g.astype(np.float64) - nrm) <= nrm_tol * scale).all(), \
        float((np.abs(nrm_g.astype(np.float64) - nrm) / scale).max())


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
    levels, total = _check_levels(levels_g, codes, L, oracle)
    assert n_g == total
    cell, code, k, edge = oracle.traverse(codes, levels, L, 0, total)
    _, pos, nrm = oracle.geometry(field, L, iso, cell, code, k, edge, normal_mode=0, extent=extent)
    _check_geometry(pos_g, nrm_g, pos, nrm, L, extent)


@pytest.mark.parametrize("lattice,cells,extent,seed", CASES[:3])
def test_binary_mode_matches_reference_glsl(oracle, lattice, cells, extent, seed):
    """HPMCsetFieldAsBinary: threshold 0.5 in the base level (shadergen.cpp:99-101),
    edge midpoints and the per-case table normals carried in the edge table's
    fractions (shadergen.cpp:507-522, constants.cpp:217-273, triface.cpp:391-399)."""
    rng = np.random.default_rng(100 + seed)
    fx, fy, fz = lattice
    field = (rng.random((fz, fy, fx)) < 0.5).astype(np.float32)  # a binary volume: 0 and 1
    levels_g, n_g, pos_g, nrm_g = _glsl().run(field, 0.25, cells=cells, extent=extent, binary=True)
    L = oracle.layout(lattice, cells)
    codes = oracle.codes(field, L, 0.25, binary=True)
    levels, total = _check_levels(levels_g, codes, L, oracle)
    assert n_g == total > 0
    cell, code, k, edge = oracle.traverse(codes, levels, L, 0, total)
    _, pos, nrm = oracle.geometry(field, L, 0.25, cell, code, k, edge, binary=True, extent=extent)
    _check_geometry(pos_g, nrm_g, pos, nrm, L, extent)


@pytest.mark.parametrize("normal_mode", [0, 2])
def test_rgba_gradient_texture_matches_reference_glsl(oracle, normal_mode):
    """HPMCsetFieldTexture3D(h, tex, gradient): an RGBA float texture whose
    alpha is the field; with gradient the normal is iso - lerp(rgb at a,
    rgb at b, t) (shadergen.cpp:260-266, 539-551), without it the forward
    differences of the alpha channel."""
    rng = np.random.default_rng(21 + normal_mode)
    fz, fy, fx = 11, 14, 13
    field = rng.normal(size=(fz, fy, fx, 4)).astype(np.float32)
    field[..., 3][rng.random((fz, fy, fx)) < 0.05] = 0.25  # ties
    iso = 0.25
    gradient = normal_mode == 2
    levels_g, n_g, pos_g, nrm_g = _glsl().run(field, iso, gradient=gradient)
    L = oracle.layout((fx, fy, fz))
    codes = oracle.codes(field, L, iso)
    assert np.array_equal(codes, oracle.codes(np.ascontiguousarray(field[..., 3]), L, iso))
    levels, total = _check_levels(levels_g, codes, L, oracle)
    assert n_g == total > 0
    cell, code, k, edge = oracle.traverse(codes, levels, L, 0, total)
    _, pos, nrm = oracle.geometry(field, L, iso, cell, code, k, edge, normal_mode=normal_mode)
    _check_geometry(pos_g, nrm_g, pos, nrm, L, (1.0, 1.0, 1.0))


def _cayley_snippet():
    import os

    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                        "cayley_fetch.glsl")
    if not os.path.exists(path):
        pytest.skip("the Cayley demo's fetch snippet is extracted by oracle/Makefile from the HPMC tree")
    with open(path) as f:
        return f.read()


@pytest.mark.parametrize("gradient", [False, True])
def test_custom_fetch_cayley_snippet_matches_reference_glsl(oracle, gradient):
    """HPMCsetFieldCustom with the Cayley demo's own GLSL (apps/cayley/cayley.cpp:75-94)
    through the reference's custom-fetch generator (shadergen.cpp:270-286) vs the
    oracle's restatement of the same functor (the product's "hpmc:cayley").  The
    shader evaluates the snippet at texel centres it derives from the tile
    coordinates, which can round differently from (i + 0.5) / n in the last
    place: the case indices must still agree (no sample lies that close to the
    iso-value here); positions within 2e-5 of the cell spacing (measured: at
    most 1.1e-5, 99 % below 3.6e-6) and normals within 2e-5 relative, both
    from the values' last-place differences at those evaluation points."""
    snippet = _cayley_snippet()
    shape = (26, 21, 24)  # (z, y, x)
    fz, fy, fx = shape
    levels_g, n_g, pos_g, nrm_g = _glsl().run(None, 0.0, custom=snippet, shape=shape, gradient=gradient)
    F = oracle.Functor("hpmc:cayley", [], shape)
    L = oracle.layout((fx, fy, fz))
    codes = oracle.codes(F, L, 0.0)
    levels, total = _check_levels(levels_g, codes, L, oracle)
    assert n_g == total > 0
    cell, code, k, edge = oracle.traverse(codes, levels, L, 0, total)
    _, pos, nrm = oracle.geometry(F, L, 0.0, cell, code, k, edge, normal_mode=2 if gradient else 0)
    _check_geometry(pos_g, nrm_g, pos, nrm, L, (1.0, 1.0, 1.0), nrm_tol=2e-5, spacing_tol=2e-5)


def test_metaballs_64_full_size_matches_reference_glsl(oracle):
    """The 64^3 metaball workload at its stated size, texture mode.  At this
    size the reference prints its 1/(2 size) = 1/512 constant inexactly
    (0.00195312): its positions differ from the lattice-exact ones by up to
    ~1e-3 cells, and exactly by that effect -- they equal the shader's tile
    arithmetic with the printed constant (tests/reference_positions.py) to FP32
    rounding, while the crossing parameter, the normals and the topology
    agree with the oracle as everywhere else."""
    from hpmc_b200 import datasets
    from tests.reference_positions import printed_texel_constant, reference_positions, shader_rounding

    field, iso = datasets.metaballs_64()
    levels_g, n_g, pos_g, nrm_g = _glsl().run(field, iso, max_vertices=1 << 18)
    L = oracle.layout((64, 64, 64))
    codes = oracle.codes(field, L, iso)
    levels, total = _check_levels(levels_g, codes, L, oracle)
    assert n_g == total > 0
    cell, code, k, edge = oracle.traverse(codes, levels, L, 0, total)
    t, pos, nrm = oracle.geometry(field, L, iso, cell, code, k, edge, normal_mode=0)
    c_printed = printed_texel_constant(oracle.ref_glsl(5, (64, 64, 64)))
    assert c_printed != 1.0 / (2 * L.size)  # the inexact constant
    pos_ref = reference_positions(L, cell, edge, t, oracle.edge_table(), c_printed)
    spacing = 1.0 / np.array(L.cells)
    assert (np.abs(pos_g - pos_ref) <= 4e-6 * (np.abs(pos_ref) + spacing) + shader_rounding(L)).all()
    off = np.abs(pos_g - pos) / spacing
    # the printed constant's effect: up to 2 size x its relative error, in cells
    assert 1e-4 < off.max() < 1.1 * 2 * L.size * abs(c_printed * 2 * L.size - 1)
    _check_geometry(pos_ref, nrm_g, pos, nrm, L, (1.0, 1.0, 1.0), pos_tol=1.0)  # normals only


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
