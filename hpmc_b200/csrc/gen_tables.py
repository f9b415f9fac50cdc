"""Build-time import of HPMC's marching-cubes case tables.

HPMC's case tables (``hpmc/src/tables.cpp``: the 256x16 triangle table in
Bourke corner order, the 12-entry edge table and the edge midpoints) are
GPL-2 data of the HPMC project.  They are read from the HPMC source tree at
build time and turned into ``_gen/hpmc_case_tables.h``; the generated header
is a build artefact (git-ignored), not part of this repository's sources.

The derivations below restate ``hpmc/src/constants.cpp``:
  * ``remap``            constants.cpp:42-50 (Bourke index -> HPMC code,
                         HPMC bit = dx + 2dy + 4dz)
  * vertex counts        constants.cpp:304-314
  * edge decode          constants.cpp:255-264 (-1 entries -> edge 0)
  * binary-field normals constants.cpp:217-252 + 266-273, evaluated in float32
                         exactly as the reference's host code does, then the
                         traversal's ``2*fract(v)-1`` (shadergen.cpp:507-510).

Usage: python gen_tables.py <hpmc source tree> <output header>
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np


def _array_body(text: str, name: str) -> str:
    m = re.search(re.escape(name) + r"\s*(\[[^=]*\])\s*=\s*\{", text)
    if not m:
        raise ValueError(f"{name} not found in tables.cpp")
    i = m.end() - 1
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i : j + 1]
    raise ValueError(f"unterminated initializer for {name}")


def _numbers(body: str) -> list[float]:
    body = re.sub(r"//[^\n]*|/\*.*?\*/", "", body, flags=re.S)
    return [float(tok.rstrip("fF")) for tok in re.findall(r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?[fF]?", body)]


def read_reference_tables(hpmc_src: str):
    path = os.path.join(hpmc_src, "hpmc", "src", "tables.cpp")
    with open(path, "r") as f:
        text = f.read()
    tri = np.array(_numbers(_array_body(text, "HPMC_triangle_table")), np.int64)
    edge = np.array(_numbers(_array_body(text, "HPMC_edge_table")), np.float32)
    mid = np.array(_numbers(_array_body(text, "HPMC_midpoint_table")), np.float32)
    if tri.size != 256 * 16 or edge.size != 12 * 4 or mid.size != 12 * 3:
        raise ValueError("unexpected table sizes in tables.cpp")
    return tri.reshape(256, 16), edge.reshape(12, 4), mid.reshape(12, 3)


def remap(c: int) -> int:
    """Bourke corner bit -> HPMC bit (dx + 2dy + 4dz)."""
    src_of_dst = (0, 1, 4, 5, 3, 2, 7, 6)
    return sum(((c >> s) & 1) << d for d, s in enumerate(src_of_dst))


def derive(tri, edge, mid):
    f32 = np.float32
    count = np.zeros(256, np.uint8)
    edge_index = np.zeros((256, 16), np.uint8)
    for j in range(256):
        r = remap(j)
        n = 0
        while n < 16 and tri[j, n] != -1:
            n += 1
        count[r] = n
        for i in range(16):
            e = int(tri[j, i])
            edge_index[r, i] = e if e >= 0 else 0
    # binary-field normals, float32 op by op
    normals = np.zeros((256, 6, 3), np.float32)
    for j in range(256):
        r = remap(j)
        for i in range(6):
            vp = []
            for k in range(3):
                ix = max(0, int(tri[j, min(15, 3 * i + k)]))
                vp.append(mid[ix])
            u = [f32(vp[2][k] - vp[0][k]) for k in range(3)]
            v = [f32(vp[1][k] - vp[0][k]) for k in range(3)]
            n = [f32(f32(u[1] * v[2]) - f32(u[2] * v[1])),
                 f32(f32(u[2] * v[0]) - f32(u[0] * v[2])),
                 f32(f32(u[0] * v[1]) - f32(u[1] * v[0]))]
            sq = f32(f32(f32(n[0] * n[0]) + f32(n[1] * n[1])) + f32(n[2] * n[2]))
            s = f32(f32(0.5) * np.sqrt(sq, dtype=np.float32))
            for k in range(3):
                tmp = f32(f32(s * n[k]) + f32(0.5))
                if tmp < 0:
                    tmp = f32(0.000001)
                if tmp >= 1:
                    tmp = f32(0.999999)
                normals[r, i, k] = tmp
    binary_normal = np.zeros((256, 16, 3), np.float32)
    for c in range(256):
        for i in range(15):
            e = edge_index[c, i]
            for k in range(3):
                val = f32(edge[e, k] + normals[c, i // 3, k])
                fr = f32(val - np.floor(val))
                binary_normal[c, i, k] = f32(f32(2.0) * fr - f32(1.0))
        for k in range(3):  # entry 15 of edge_decode_normal is 0 -> 2*0-1
            binary_normal[c, 15, k] = f32(-1.0)
    return count, edge_index, binary_normal


def emit(out_path: str, tri, edge, mid) -> None:
    count, edge_index, binary_normal = derive(tri, edge, mid)
    packed_edges = 0
    for e in range(12):
        sx, sy, sz, ax = (int(edge[e, 0]), int(edge[e, 1]), int(edge[e, 2]), int(edge[e, 3]))
        packed_edges |= (sx | (sy << 1) | (sz << 2) | (ax << 3)) << (5 * e)
    edge_words = []
    for c in range(256):
        w = 0
        for k in range(16):
            w |= int(edge_index[c, k]) << (4 * k)
        edge_words.append(w)
    lines = [
        "// Generated at build time by gen_tables.py from HPMC's hpmc/src/tables.cpp",
        "// (GPL-2 data of the HPMC project).  Build artefact: not committed, do not edit.",
        "#pragma once",
        "#include <stdint.h>",
        "// vertices per HPMC code (bit dx+2dy+4dz set iff f < iso)",
        "#define HPMC_GEN_VERTEX_COUNT { " + ", ".join(str(int(v)) for v in count) + " }",
        "// per HPMC code: MC edge (0..11) of vertex k in nibble k",
        "#define HPMC_GEN_EDGE_NIBBLES { " + ", ".join(f"0x{w:016x}ull" for w in edge_words) + " }",
        "// per MC edge e, bits [5e, 5e+5): shift x | y<<1 | z<<2 | axis<<3",
        f"#define HPMC_GEN_EDGE_GEOMETRY 0x{packed_edges:016x}ull",
        "// binary-field normals 2*fract(edge_decode_normal.xyz)-1 per (code, k)",
        "#define HPMC_GEN_BINARY_NORMALS { "
        + ", ".join(np.format_float_scientific(float(v), unique=True) + "f" for v in binary_normal.reshape(-1))
        + " }",
        "",
    ]
    os.makedirs(os.path.dirname(os.path.abspath(out_path)), exist_ok=True)
    tmp = out_path + ".tmp"
    with open(tmp, "w") as f:
        f.write("\n".join(lines))
    os.replace(tmp, out_path)


def main(argv):
    if len(argv) != 3:
        print(__doc__)
        return 2
    tri, edge, mid = read_reference_tables(argv[1])
    emit(argv[2], tri, edge, mid)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
