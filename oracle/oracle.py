"""ctypes binding of the test oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/_ref/libhpmc_oracle.so`` (CPU restatement of HPMC's
HistoPyramid marching cubes, see ``hpmc_oracle.h``) and
``oracle/_ref/libhpmc_ref.so`` (the reference's own layout, tables and GLSL
generator compiled from the HPMC sources).  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs import this module; the
product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF_DIR = os.path.join(_HERE, "_ref")

F32, U8, UNORM8, F64, FUNCTOR, F32X4 = 0, 1, 2, 3, 4, 5  # F64: geometry and adjoint only
# F32X4: (z, y, x, 4) float32 = gradient x, y, z and the value (a GL RGBA texture)
NORMALS_FORWARD, NORMALS_CENTRAL = 0, 1
# analytic-gradient normals of a functor field: the reference's iso - lerp(grad), or -lerp(grad)
NORMALS_GRADIENT, NORMALS_GRADIENT_CENTRAL = 2, 3


def build(hpmc_src: str | None = None) -> None:
    """Run the oracle's Makefile (needs the HPMC source tree)."""
    import subprocess

    cmd = ["make", "-s", "-C", _HERE]
    if hpmc_src:
        cmd.append(f"HPMC_SRC={hpmc_src}")
    subprocess.run(cmd, check=True)


class _Layout(C.Structure):
    _fields_ = [
        ("lattice", C.c_int * 3),
        ("cells", C.c_int * 3),
        ("tile", C.c_int * 2),
        ("layout", C.c_int * 2),
        ("size_l2", C.c_int),
        ("size", C.c_int),
    ]


@dataclass(frozen=True)
class Layout:
    lattice: tuple
    cells: tuple
    tile: tuple
    layout: tuple
    size_l2: int
    size: int

    def level_entries(self, j: int) -> int:
        e = self.size_l2 + 1 - j
        return 1 if e <= 0 else 1 << (2 * e)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_REF_DIR, "libhpmc_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} missing (run make -C oracle)")
        L = C.CDLL(path)
        vp, ip, fp, u8p = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_uint8)
        L.oracle_layout.argtypes = [ip, ip, C.POINTER(_Layout)]
        L.oracle_layout.restype = C.c_int
        L.oracle_remap_code.argtypes = [C.c_int]
        L.oracle_remap_code.restype = C.c_int
        L.oracle_tables.argtypes = [vp, vp, vp, vp]
        L.oracle_codes.argtypes = [vp, C.c_int, C.POINTER(_Layout), C.c_size_t, C.c_size_t,
                                   C.c_float, C.c_int, vp]
        L.oracle_cell_key.argtypes = [C.POINTER(_Layout), C.c_int, C.c_int, C.c_int]
        L.oracle_cell_key.restype = C.c_uint64
        L.oracle_level_entries.argtypes = [C.POINTER(_Layout), C.c_int]
        L.oracle_level_entries.restype = C.c_uint64
        L.oracle_pyramid.argtypes = [C.POINTER(_Layout), vp, vp, C.POINTER(C.c_void_p)]
        L.oracle_pyramid.restype = C.c_uint64
        L.oracle_level0_texture.argtypes = [C.POINTER(_Layout), vp, vp, vp]
        L.oracle_traverse.argtypes = [C.POINTER(_Layout), vp, C.POINTER(C.c_void_p), vp,
                                      C.c_uint64, C.c_uint64, vp, vp, vp, vp]
        L.oracle_geometry.argtypes = [vp, C.c_int, C.POINTER(_Layout), C.c_size_t, C.c_size_t,
                                      C.c_float, C.c_int, C.c_int, fp, vp, C.c_uint64, vp, vp,
                                      vp, vp, vp, vp, vp]
        L.oracle_extract.argtypes = [vp, C.c_int, ip, ip, C.c_float, C.c_int, C.c_int, fp, vp,
                                     vp, C.c_uint64, C.c_int]
        L.oracle_extract.restype = C.c_uint64
        L.oracle_max_threads.restype = C.c_int
        L.oracle_edge_table.argtypes = [vp]
        L.oracle_adjoint.argtypes = [vp, C.c_int, C.POINTER(_Layout), C.c_size_t, C.c_size_t, C.c_float, C.c_int,
                                     fp, C.c_uint64, vp, vp, vp, vp, vp, vp]
        _lib = L
    return _lib


def ref():
    """The reference's own compiled code (layout, tables, GLSL generator)."""
    global _ref
    if _ref is None:
        path = os.path.join(_REF_DIR, "libhpmc_ref.so")
        if not os.path.exists(path):
            raise RuntimeError(f"reference harness not built: {path} missing")
        R = C.CDLL(path)
        ip = C.POINTER(C.c_int)
        R.hpmc_ref_layout.argtypes = [C.c_int] * 6 + [ip]
        R.hpmc_ref_layout.restype = C.c_int
        R.hpmc_ref_triangle_table.restype = C.POINTER(C.c_int)
        R.hpmc_ref_edge_table.restype = C.POINTER(C.c_float)
        R.hpmc_ref_midpoint_table.restype = C.POINTER(C.c_float)
        R.hpmc_ref_glsl.argtypes = [C.c_int, ip, ip, C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int]
        R.hpmc_ref_glsl.restype = C.c_void_p
        R.hpmc_ref_glsl_custom.argtypes = [C.c_int, ip, ip, C.POINTER(C.c_float), C.c_int, C.c_int, C.c_int,
                                           C.c_char_p]
        R.hpmc_ref_glsl_custom.restype = C.c_void_p
        R.hpmc_ref_free.argtypes = [C.c_void_p]
        _ref = R
    return _ref


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class _FunctorParams(C.Structure):
    _fields_ = [("id", C.c_int), ("count", C.c_int), ("p", C.c_float * 136)]


class Functor:
    """A field functor on a lattice of `shape` (z, y, x): the oracle's form of
    HPMCsetFieldCustom + HPMCsetBuilderUniforms (hpiface.cpp:187-222)."""

    IDS = {"hpmc:cayley": 1, "hpmc:metaballs": 2, "hpmc:twist_metaballs": 3, "hpmc:spheres": 4,
           "app:torus": 5}  # app:torus: the caller-registered functor of hpmc_b200/apps/custom_functor.cu

    def __init__(self, name: str, params, shape):
        self.name = name
        self.shape = tuple(int(v) for v in shape)
        self.params = [float(v) for v in params]
        self.c = _FunctorParams()
        self.c.id = self.IDS[name]
        self.c.count = len(self.params)
        for i, v in enumerate(self.params):
            self.c.p[i] = v


def _field(field, unorm=False):
    """(pointer, type, contiguous field) of an array or a Functor."""
    if isinstance(field, Functor):
        return C.cast(C.pointer(field.c), C.c_void_p), FUNCTOR, field
    field = np.ascontiguousarray(field)
    return _ptr(field), _field_type(field, unorm), field


def _to_layout(s: _Layout) -> Layout:
    return Layout(tuple(s.lattice), tuple(s.cells), tuple(s.tile), tuple(s.layout), s.size_l2, s.size)


def layout(lattice, cells=None):
    lattice = [int(v) for v in lattice]
    cells = [v - 1 for v in lattice] if cells is None else [int(v) for v in cells]
    s = _Layout()
    ok = lib().oracle_layout((C.c_int * 3)(*lattice), (C.c_int * 3)(*cells), C.byref(s))
    return _to_layout(s) if ok else None


def _struct(L: Layout) -> _Layout:
    s = _Layout()
    s.lattice[:] = list(L.lattice)
    s.cells[:] = list(L.cells)
    s.tile[:] = list(L.tile)
    s.layout[:] = list(L.layout)
    s.size_l2 = L.size_l2
    s.size = L.size
    return s


def ref_layout(lattice, cells=None):
    lattice = [int(v) for v in lattice]
    cells = [v - 1 for v in lattice] if cells is None else [int(v) for v in cells]
    out = (C.c_int * 6)()
    if not ref().hpmc_ref_layout(*lattice, *cells, out):
        return None
    return tuple(out)


def ref_tables():
    R = ref()
    tri = np.ctypeslib.as_array(R.hpmc_ref_triangle_table(), shape=(256, 16)).copy()
    edge = np.ctypeslib.as_array(R.hpmc_ref_edge_table(), shape=(12, 4)).copy()
    mid = np.ctypeslib.as_array(R.hpmc_ref_midpoint_table(), shape=(12, 3)).copy()
    return tri, edge, mid


def ref_glsl(which: int, lattice, cells=None, extent=(1.0, 1.0, 1.0), binary=False,
             gradient=False, gl_target=9, custom_source: str | None = None) -> str:
    """GLSL text the reference generates (which: 0 defines, 1 fetch, 2 base
    level, 3 first reduction, 4 upper reduction, 5 extract vertex); with
    custom_source, for the custom-fetch mode with that application snippet."""
    lattice = [int(v) for v in lattice]
    cells = [v - 1 for v in lattice] if cells is None else [int(v) for v in cells]
    args = (which, (C.c_int * 3)(*lattice), (C.c_int * 3)(*cells), (C.c_float * 3)(*extent), int(binary),
            int(gradient), int(gl_target))
    if custom_source is None:
        p = ref().hpmc_ref_glsl(*args)
    else:
        p = ref().hpmc_ref_glsl_custom(*args, custom_source.encode())
    if not p:
        raise ValueError("layout rejected")
    s = C.string_at(p).decode()
    ref().hpmc_ref_free(p)
    return s


def tables():
    count = np.zeros(256, np.uint8)
    eidx = np.zeros(256 * 16, np.uint8)
    ed = np.zeros(256 * 16 * 4, np.float32)
    edn = np.zeros(256 * 16 * 4, np.float32)
    lib().oracle_tables(_ptr(count), _ptr(eidx), _ptr(ed), _ptr(edn))
    return count, eidx.reshape(256, 16), ed.reshape(256, 16, 4), edn.reshape(256, 16, 4)


def _field_type(field: np.ndarray, unorm: bool) -> int:
    if field.dtype == np.float32 and field.ndim == 4 and field.shape[3] == 4:
        return F32X4
    if field.dtype == np.float32:
        return F32
    if field.dtype == np.float64:
        return F64
    if field.dtype == np.uint8:
        return UNORM8 if unorm else U8
    raise TypeError(f"unsupported field dtype {field.dtype}")


def codes(field: np.ndarray, L: Layout, iso: float, binary=False, unorm=False) -> np.ndarray:
    """Per-cell MC codes, shape (cz, cy, cx). field is C-contiguous (fz, fy, fx)."""
    fptr, ftype, field = _field(field, unorm)
    cx, cy, cz = L.cells
    out = np.zeros((cz, cy, cx), np.uint8)
    fx, fy, _ = L.lattice
    s = _struct(L)
    lib().oracle_codes(fptr, ftype, C.byref(s), fx, fx * fy, float(iso), int(binary), _ptr(out))
    return out


def pyramid(codes_arr: np.ndarray, L: Layout):
    """Compact levels j = 0..size_l2+1 (uint32) and the total vertex count."""
    count, _, _, _ = tables()
    levels = [np.zeros(L.level_entries(j), np.uint32) for j in range(L.size_l2 + 2)]
    ptrs = (C.c_void_p * len(levels))(*[lv.ctypes.data for lv in levels])
    s = _struct(L)
    total = lib().oracle_pyramid(C.byref(s), _ptr(np.ascontiguousarray(codes_arr)), _ptr(count), ptrs)
    return levels, int(total)


def level0_texture(codes_arr: np.ndarray, L: Layout) -> np.ndarray:
    count, _, _, _ = tables()
    tex = np.zeros((L.size, L.size, 4), np.float32)
    s = _struct(L)
    lib().oracle_level0_texture(C.byref(s), _ptr(np.ascontiguousarray(codes_arr)), _ptr(count), _ptr(tex))
    return tex


def traverse(codes_arr, levels, L: Layout, v0: int, v1: int):
    _, eidx, _, _ = tables()
    n = v1 - v0
    cell = np.zeros((n, 3), np.int32)
    code = np.zeros(n, np.uint8)
    k = np.zeros(n, np.uint8)
    edge = np.zeros(n, np.uint8)
    ptrs = (C.c_void_p * len(levels))(*[lv.ctypes.data for lv in levels])
    s = _struct(L)
    lib().oracle_traverse(C.byref(s), _ptr(np.ascontiguousarray(codes_arr)), ptrs,
                          _ptr(np.ascontiguousarray(eidx.reshape(-1))), v0, v1, _ptr(cell),
                          _ptr(code), _ptr(k), _ptr(edge))
    return cell, code, k, edge


def geometry(field, L: Layout, iso, cell, code, k, edge, *, binary=False,
             normal_mode=NORMALS_FORWARD, extent=(1.0, 1.0, 1.0), unorm=False):
    fptr, ftype, field = _field(field, unorm)
    _, _, _, edn = tables()
    n = len(edge)
    t = np.zeros(n, np.float64)
    pos = np.zeros((n, 3), np.float64)
    nrm = np.zeros((n, 3), np.float64)
    fx, fy, _ = L.lattice
    s = _struct(L)
    ext = (C.c_float * 3)(*extent)
    lib().oracle_geometry(fptr, ftype, C.byref(s), fx, fx * fy,
                          float(iso), int(binary), int(normal_mode), ext,
                          _ptr(np.ascontiguousarray(edn.reshape(-1))), n,
                          _ptr(np.ascontiguousarray(cell)), _ptr(np.ascontiguousarray(code)),
                          _ptr(np.ascontiguousarray(k)), _ptr(np.ascontiguousarray(edge)),
                          _ptr(t), _ptr(pos), _ptr(nrm))
    return t, pos, nrm


def adjoint(field, L: Layout, iso, cell, edge, dpos, dnrm, *, normal_mode=NORMALS_FORWARD,
            extent=(1.0, 1.0, 1.0), unorm=False, with_abs=False):
    """FP64 dL/df of L = sum dpos.p + dnrm.n over the vertices (cell, edge);
    dpos, dnrm are (n, 3).  Returns an array of the field's shape (float64),
    and with_abs also the per-sample sum of |terms|."""
    field = np.ascontiguousarray(field)
    n = len(edge)
    fx, fy, _ = L.lattice
    s = _struct(L)
    out = np.zeros(field.shape, np.float64)
    absum = np.zeros(field.shape, np.float64) if with_abs else None
    lib().oracle_adjoint(_ptr(field), _field_type(field, unorm), C.byref(s), fx, fx * fy, float(iso),
                         int(normal_mode), (C.c_float * 3)(*extent), n, _ptr(np.ascontiguousarray(cell)),
                         _ptr(np.ascontiguousarray(edge)),
                         _ptr(np.ascontiguousarray(dpos, dtype=np.float64)),
                         _ptr(np.ascontiguousarray(dnrm, dtype=np.float64)), _ptr(out),
                         _ptr(absum) if with_abs else None)
    return (out, absum) if with_abs else out


def cell_key(L: Layout, x: int, y: int, z: int) -> int:
    s = _struct(L)
    return int(lib().oracle_cell_key(C.byref(s), x, y, z))


def extract_count(field, iso, cells=None, *, binary=False, normal_mode=NORMALS_FORWARD,
                  extent=(1.0, 1.0, 1.0), unorm=False, threads=0, geometry=False):
    """Whole CPU extraction (the CPU baseline).  Returns (count, pos, nrm)."""
    field = np.ascontiguousarray(field)
    lattice = [field.shape[2], field.shape[1], field.shape[0]]
    cells = [v - 1 for v in lattice] if cells is None else list(cells)
    cap = 0
    pos = nrm = None
    if geometry:
        L = layout(lattice, cells)
        lv, total = pyramid(codes(field, L, iso, binary, unorm), L)
        cap = total
        pos = np.zeros((max(cap, 1), 3), np.float32)
        nrm = np.zeros((max(cap, 1), 3), np.float32)
    n = lib().oracle_extract(_ptr(field), _field_type(field, unorm), (C.c_int * 3)(*lattice),
                             (C.c_int * 3)(*cells), float(iso), int(binary), int(normal_mode),
                             (C.c_float * 3)(*extent), _ptr(pos) if pos is not None else None,
                             _ptr(nrm) if nrm is not None else None, cap, int(threads))
    if geometry:
        return int(n), pos[:n], nrm[:n]
    return int(n), None, None


def edge_table() -> np.ndarray:
    """The reference's edge table, (12, 4): first-corner shift x, y, z and axis."""
    out = np.zeros(48, np.float32)
    lib().oracle_edge_table(_ptr(out))
    return out.reshape(12, 4)


def max_threads() -> int:
    return int(lib().oracle_max_threads())
