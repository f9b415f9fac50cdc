"""Positions as the reference's extraction shader computes them.

The reference's vertex shader (shadergen.cpp:497-503, 512-520, 553-560)
recovers a vertex's cell from its texel position through the constant
1/(2 size), which the shader generator prints through a default-precision
C++ stream, i.e. with 6 significant digits (0.00195312 for 1/512).  For
pyramids of 256 texels and more that constant is inexact, and every position
inherits its relative error through the tile coordinate: up to about
2 size x 6e-6 cells.  Slice, edge and crossing parameter are unaffected (the
error stays far below half a texel).

This module restates that arithmetic (in FP64) from the oracle's cell, edge
and crossing parameter and the constant read from the generated text, so a
test can check that the reference's positions differ from the lattice-exact
ones by exactly this effect.  The product and the oracle compute
lattice-exact positions (lattice index x extent / cells).
"""
from __future__ import annotations

import re

import numpy as np


def printed_texel_constant(extract_glsl: str) -> float:
    """The 1/(2 size) constant as the generated extraction shader prints it."""
    m = re.search(r"vec2 bar = ([0-9.eE+-]+)\*baz;", extract_glsl)
    if not m:
        raise ValueError("constant not found in the extraction shader")
    return float(m.group(1))


def shader_rounding(L, extent=(1.0, 1.0, 1.0)):
    """Per-axis absolute bound of the FP32 rounding in the shader's tile
    arithmetic: fract(foo) with foo up to the number of tiles loses up to an
    ulp of that many tiles, scaled to world units by 2 tile / cells (x, y);
    a few such ulps, as the position is rescaled twice afterwards."""
    eps = 2.0 ** -24
    cx, cy, _ = L.cells
    tx, ty = L.tile
    lx, ly = L.layout
    return np.array([8 * eps * lx * 2 * tx * extent[0] / cx, 8 * eps * ly * 2 * ty * extent[1] / cy, 0.0])


def reference_positions(L, cell, edge, t, edge_table, c_printed, extent=(1.0, 1.0, 1.0)):
    """(n, 3) positions of vertices (cell (x, y, z), MC edge, t) through the
    shader's tile arithmetic with the printed constant."""
    fx, fy, _ = L.lattice
    cx, cy, cz = L.cells
    tx, ty = L.tile
    lx, ly = L.layout
    x = cell[:, 0].astype(np.float64)
    y = cell[:, 1].astype(np.float64)
    z = cell[:, 2].astype(np.int64)
    # virtual cell coordinates (shadergen.cpp:103-104): slice tile (z mod Lx, z div Lx)
    X = 2.0 * tx * (z % lx) + x
    Y = 2.0 * ty * (z // lx) + y
    foo_x = lx * (c_printed * (X + 0.5))
    foo_y = ly * (c_printed * (Y + 0.5))
    tp_x = (2.0 * tx / fx) * (foo_x - np.floor(foo_x))
    tp_y = (2.0 * ty / fy) * (foo_y - np.floor(foo_y))
    slice_ = np.floor(foo_x) + lx * np.floor(foo_y)
    e = edge_table[edge]
    shift, axis = e[:, :3], e[:, 3].astype(np.int64)
    pa = np.stack([tp_x + shift[:, 0] / fx, tp_y + shift[:, 1] / fy, slice_ + shift[:, 2]], 1)
    step = np.zeros_like(pa)
    step[np.arange(len(axis)), axis] = 1.0
    step[:, 0] /= fx
    step[:, 1] /= fy
    p = pa + t[:, None] * step
    p[:, 0] -= 0.5 / fx
    p[:, 1] -= 0.5 / fy
    p *= np.array([extent[0] * fx / cx, extent[1] * fy / cy, extent[2] / cz])
    return p
