"""TEST INFRASTRUCTURE: run the reference's own generated GLSL on the CPU.

The reference generates every pass of the HistoPyramid as GLSL text
(hpmc/src/shadergen.cpp) and runs it in a GL driver; there is no GL stack on
this machine.  This module takes that text -- produced by the reference's
shader generator compiled from the HPMC tree (oracle/_ref/libhpmc_ref.so,
see oracle/Makefile) -- rewrites the few constructs C++ does not share with
GLSL (uniform declarations, float literals, swizzles, `out` parameters, the
name `main`), compiles it against oracle/glsl_emu.hpp with the host compiler,
and drives the passes the way buildpass.cpp:42-178 and triface.cpp:332-457 do
(GL 3 targets): base level, first reduction (floor filter), upper reductions,
then extractVertex for every vertex id.  Field modes: a Texture3D field
(alpha texture, or an RGBA float texture whose .xyz the gradient mode reads),
or the custom-fetch mode with an application's GLSL snippet
(HPMCsetFieldCustom); binary fields bind the edge table with table normals
(triface.cpp:391-399).

The outputs (every mip level, the vertex count, positions and normals in
FP32 GLSL arithmetic) pin the oracle's restatement to the reference's code.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import re
import shutil
import subprocess

import numpy as np

from . import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref", "glsl")

_FLOAT = re.compile(r"(?<![\w.])(\d+\.\d*(?:[eE][-+]?\d+)?|\.\d+(?:[eE][-+]?\d+)?)(?![\w.])")


def translate(text: str) -> str:
    """GLSL (the subset the reference emits) -> C++ against glsl_emu.hpp."""
    out = []
    for line in text.splitlines():
        if line.strip().startswith("uniform "):
            continue  # declared by the harness per pass
        if line.startswith("#"):
            out.append(line)
            continue
        line = _FLOAT.sub(lambda m: m.group(1) + "f", line)
        line = re.sub(r"\.(xyz|xy)(?![\w(])", r".\1()", line)
        line = re.sub(r"\.a(?![\w(])", r".a()", line)
        line = re.sub(r"\bout\s+(\w+)\s+(\w+)", r"\1& \2", line)
        line = re.sub(r"\bmain\s*\(", "shader_main(", line)
        out.append(line)
    return "\n".join(out) + "\n"


_DRIVER = r"""
#include <omp.h>
extern "C" int glsl_run(const float* field, int rgba, int fx, int fy, int fz, float iso, int size, int size_l2,
                        const float* count_rgba, const float* edge_rgba, float* mips, int max_vertices,
                        float* pos, float* nrm, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    // --- base level (buildpass.cpp:62-92): one fragment per texel, texcoord at its centre
    std::vector<std::vector<float>> mip(size_l2 + 1);
    mip[0].assign((size_t)size * size * 4, 0.f);
    sampler3D field_tex;
    if (rgba) field_tex.rgba = field; else field_tex.alpha = field;
    field_tex.nx = fx; field_tex.ny = fy; field_tex.nz = fz;
    sampler1D count_tex;
    count_tex.rgba = count_rgba; count_tex.n = 256;
#pragma omp parallel
    {
        sh_base::HPMC_scalarfield = field_tex;  // uniforms: once per thread
        sh_base::HPMC_vertex_count = count_tex;
        sh_base::HPMC_threshold = iso;
#pragma omp for schedule(static)
    for (int j = 0; j < size; j++) {
        for (int i = 0; i < size; i++) {
            sh_base::gl_TexCoord[0] = vec4((i + 0.5f) / (float)size, (j + 0.5f) / (float)size, 0.f, 1.f);
            sh_base::shader_main();
            float* t = &mip[0][4 * ((size_t)j * size + i)];
            t[0] = sh_base::gl_FragColor.x; t[1] = sh_base::gl_FragColor.y;
            t[2] = sh_base::gl_FragColor.z; t[3] = sh_base::gl_FragColor.w;
        }
    }
    }
    // --- reductions (buildpass.cpp:104-159): first with the floor filter
    for (int m = 1; m <= size_l2; m++) {
        const int w = size >> m;
        mip[m].assign((size_t)w * w * 4, 0.f);
        sampler2D hp;
        for (int l = 0; l < m; l++) { hp.levels.push_back(mip[l].data()); hp.w.push_back(size >> l); hp.h.push_back(size >> l); }
#pragma omp parallel
        {
            sh_first::HPMC_histopyramid = hp; sh_first::HPMC_src_level = 0;
            sh_upper::HPMC_histopyramid = hp; sh_upper::HPMC_src_level = m - 1;
#pragma omp for schedule(static)
        for (int j = 0; j < w; j++) {
            for (int i = 0; i < w; i++) {
                vec4 c;
                if (m == 1) {
                    sh_first::gl_FragCoord = vec4(i + 0.5f, j + 0.5f, 0.f, 1.f);
                    sh_first::shader_main(); c = sh_first::gl_FragColor;
                } else {
                    sh_upper::gl_FragCoord = vec4(i + 0.5f, j + 0.5f, 0.f, 1.f);
                    sh_upper::shader_main(); c = sh_upper::gl_FragColor;
                }
                float* t = &mip[m][4 * ((size_t)j * w + i)];
                t[0] = c.x; t[1] = c.y; t[2] = c.z; t[3] = c.w;
            }
        }
        }
    }
    size_t off = 0;
    if (mips)
        for (int m = 0; m <= size_l2; m++) {
            std::copy(mip[m].begin(), mip[m].end(), mips + off);
            off += mip[m].size();
        }
    // --- count (hpiface.cpp:323-327)
    const float* top = mip[size_l2].data();
    const int N = (int)(std::floor(top[0]) + std::floor(top[1]) + std::floor(top[2]) + std::floor(top[3]));
    // --- extraction (triface.cpp:423-428): extractVertex per vertex id
    sampler2D hp;
    for (int l = 0; l <= size_l2; l++) { hp.levels.push_back(mip[l].data()); hp.w.push_back(size >> l); hp.h.push_back(size >> l); }
    sampler2D et; et.levels.push_back(edge_rgba); et.w.push_back(16); et.h.push_back(256);
    const int nv = N < max_vertices ? N : max_vertices;
#pragma omp parallel
    {
        sh_ext::HPMC_histopyramid = hp; sh_ext::HPMC_edge_table = et;
        sh_ext::HPMC_scalarfield = field_tex;
        sh_ext::HPMC_threshold = iso; sh_ext::HPMC_key_offset = 0.f;
#pragma omp for schedule(static)
    for (int v = 0; v < nv; v++) {
        sh_ext::gl_VertexID = v;
        vec3 p, n;
        sh_ext::extractVertex(p, n);
        pos[3 * (size_t)v] = p.x; pos[3 * (size_t)v + 1] = p.y; pos[3 * (size_t)v + 2] = p.z;
        nrm[3 * (size_t)v] = n.x; nrm[3 * (size_t)v + 1] = n.y; nrm[3 * (size_t)v + 2] = n.z;
    }
    }
    return N;
}
"""


def program(lattice, cells=None, extent=(1.0, 1.0, 1.0), binary=False, gradient=False,
            custom: str | None = None) -> str:
    """C++ source of the reference's passes for one configuration (custom:
    the application's GLSL fetch snippet of the custom-fetch mode)."""
    g = lambda which: O.ref_glsl(which, lattice, cells, extent, binary=binary, gradient=gradient,  # noqa: E731
                                 custom_source=custom)
    defines, fetch = g(0), translate(g(1))
    parts = ['#include "glsl_emu.hpp"', "#include <algorithm>", "using namespace glsl;", translate(defines)]
    # uniforms and built-ins are per-thread: the harness runs fragments and
    # vertices in parallel (OpenMP), one shader invocation per thread at a time
    parts.append("namespace sh_base {\nthread_local sampler3D HPMC_scalarfield; thread_local sampler1D HPMC_vertex_count;\n"
                 "thread_local float HPMC_threshold;\nthread_local vec4 gl_FragColor; thread_local vec4 gl_TexCoord[1];\n"
                 + fetch + translate(g(2)) + "}")
    for ns, which in (("sh_first", 3), ("sh_upper", 4)):
        parts.append(f"namespace {ns} {{\nthread_local sampler2D HPMC_histopyramid; thread_local int HPMC_src_level;\n"
                     "thread_local vec2 HPMC_delta;\nthread_local vec4 gl_FragColor; thread_local vec4 gl_FragCoord;\n"
                     + translate(g(which)) + "}")
    parts.append("namespace sh_ext {\nthread_local sampler3D HPMC_scalarfield; thread_local sampler2D HPMC_histopyramid;\n"
                 "thread_local sampler2D HPMC_edge_table; thread_local float HPMC_key_offset;\n"
                 "thread_local float HPMC_threshold; thread_local int gl_VertexID;\n" + fetch + translate(g(5)) + "}")
    parts.append(_DRIVER)
    return "\n".join(parts)


def build(lattice, cells=None, extent=(1.0, 1.0, 1.0), binary=False, gradient=False,
          custom: str | None = None) -> str:
    """Compile the passes of one configuration into a shared library (cached)."""
    src = program(lattice, cells, extent, binary, gradient, custom)
    key = hashlib.sha1((src + open(os.path.join(HERE, "glsl_emu.hpp")).read()).encode()).hexdigest()[:16]
    os.makedirs(OUT, exist_ok=True)
    so = os.path.join(OUT, f"glsl_{key}.so")
    if not os.path.exists(so):
        cpp = os.path.join(OUT, f"glsl_{key}.cpp")
        with open(cpp, "w") as f:
            f.write(src)
        cxx = shutil.which("g++") or "/usr/bin/g++"
        r = subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
                            "-I" + HERE, cpp, "-o", so + ".tmp"], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"GLSL translation did not compile:\n{r.stderr[:4000]}")
        os.replace(so + ".tmp", so)
    return so


def run(field: np.ndarray | None, iso: float, cells=None, extent=(1.0, 1.0, 1.0), max_vertices: int = 1 << 20,
        threads: int = 0, keep_levels: bool = True, *, binary=False, gradient=False, custom: str | None = None,
        shape=None):
    """The reference's passes on `threads` host threads (0: all).  `field`:
    a float (z, y, x) array bound as an alpha texture, a (z, y, x, 4) array
    bound as an RGBA float texture (gradient = True reads its .xyz), or None
    with `custom` (the custom-fetch snippet) and `shape` = (z, y, x).
    Returns (mip levels as (w, w, 4) arrays -- empty unless keep_levels --,
    vertex count, positions (n, 3), normals (n, 3)), all FP32 as the shaders
    compute them."""
    fz, fy, fx = (shape if field is None else field.shape[:3])
    lattice = (fx, fy, fz)
    L = O.layout(lattice, cells)
    lib = C.CDLL(build(lattice, cells, extent, binary, gradient, custom))
    count, _, ed, edn = O.tables()
    count_rgba = np.zeros((256, 4), np.float32)
    count_rgba[:, 3] = count
    # binary fields: the table with normals in the fractions (triface.cpp:391-399)
    edge_rgba = np.ascontiguousarray((edn if binary else ed).reshape(256, 16, 4).astype(np.float32))
    size, l2 = L.size, L.size_l2
    mips_len = sum((size >> m) ** 2 * 4 for m in range(l2 + 1))
    mips = np.zeros(mips_len if keep_levels else 1, np.float32)
    pos = np.zeros((max_vertices, 3), np.float32)
    nrm = np.zeros((max_vertices, 3), np.float32)
    f = np.zeros(4, np.float32) if field is None else np.ascontiguousarray(field, dtype=np.float32)
    rgba = int(field is not None and field.ndim == 4)
    fn = lib.glsl_run
    fn.restype = C.c_int
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    threads = int(threads) if threads and threads > 0 else (os.cpu_count() or 1)
    n = fn(p(f), rgba, fx, fy, fz, C.c_float(iso), size, l2, p(count_rgba), p(edge_rgba),
           p(mips) if keep_levels else None, max_vertices, p(pos), p(nrm), threads)
    levels, off = [], 0
    for m in range(l2 + 1 if keep_levels else 0):
        w = size >> m
        levels.append(mips[off:off + w * w * 4].reshape(w, w, 4))
        off += w * w * 4
    return levels, n, pos[:min(n, max_vertices)], nrm[:min(n, max_vertices)]
