"""hpmc_b200 -- B200-native HistoPyramid marching cubes behind HPMC's C API.

The product is the sm_100a library ``_lib/libhpmc_b200.so`` (C ABI:
``include/hpmc.h``).  This module is the host-side mirror of the reference's
operator interface for Python callers: the same handles and calls as
``hpmc/include/hpmc.h`` (constants -> HistoPyramid -> traversal handle,
build, acquire count, extract), taking torch CUDA tensors for device memory.
All computation happens in the library's kernels.

Field tensors are laid out (z, y, x) -- x fastest -- like a GL 3-D texture.
"""
from __future__ import annotations

import ctypes as C

from . import _capi
from ._capi import (NORMALS_CENTRAL, NORMALS_FORWARD, SCALAR_F32, SCALAR_F32X4, SCALAR_U8,  # noqa: F401
                    SCALAR_UNORM8, STATUS_NAMES)

__all__ = [
    "Constants", "HistoPyramid", "TraversalHandle", "Batch", "HPMCError", "extract", "lib",
    "register_device_field", "unregister_device_field",
    "NORMALS_FORWARD", "NORMALS_CENTRAL", "SCALAR_F32", "SCALAR_U8", "SCALAR_UNORM8", "SCALAR_F32X4",
]


def lib():
    return _capi.lib()


class HPMCError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}")


def _check(status: int, what: str) -> None:
    if status != _capi.OK:
        raise HPMCError(status, what)


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def _scalar_type(t, unorm: bool) -> int:
    import torch

    if t.dtype == torch.float32 and t.dim() == 4 and t.shape[3] == 4:
        return SCALAR_F32X4  # (z, y, x, 4): gradient x, y, z and the value, a GL RGBA float texture
    if t.dtype == torch.float32:
        return SCALAR_F32
    if t.dtype == torch.uint8:
        return SCALAR_UNORM8 if unorm else SCALAR_U8
    raise TypeError(f"unsupported field dtype {t.dtype} (float32 or uint8)")


def _field_layout(field) -> None:
    if not field.is_cuda:
        raise ValueError("field must be a CUDA tensor")
    if field.dim() == 4:
        if field.shape[3] != 4 or field.stride(3) != 1 or field.stride(2) != 4:
            raise ValueError("a (z, y, x, 4) field must be contiguous along x and its 4 channels")
    elif field.stride(2) != 1:
        raise ValueError("field must have unit stride along x")


def register_device_field(field, unorm: bool = False) -> int:
    """HPMCregisterDeviceField: a name for a (z, y, x) or (z, y, x, 4) CUDA
    tensor, the stand-in for a GL 3-D texture name (HPMCsetFieldTexture3D).
    The tensor must outlive its use."""
    _field_layout(field)
    es = field.element_size()
    fz, fy, fx = field.shape[:3]
    name = lib().HPMCregisterDeviceField(field.data_ptr(), _scalar_type(field, unorm), fx, fy, fz,
                                         field.stride(1) * es, field.stride(0) * es)
    if not name:
        raise HPMCError(_capi.ERR_INVALID_VALUE, "HPMCregisterDeviceField")
    return int(name)


def unregister_device_field(name: int) -> None:
    lib().HPMCunregisterDeviceField(int(name))


class Constants:
    """HPMCcreateConstants (hpmc.h:310-311): device tables for the current device."""

    def __init__(self, max_gl_major: int = 4, max_gl_minor: int = 3):
        self.ptr = lib().HPMCcreateConstants(max_gl_major, max_gl_minor)
        if not self.ptr:
            raise HPMCError(_capi.ERR_CUDA, "HPMCcreateConstants (no usable CUDA device)")

    def close(self):
        if self.ptr:
            lib().HPMCdestroyConstants(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HistoPyramid:
    """HPMCcreateHistoPyramid and the per-volume setters (hpmc.h:330-469)."""

    def __init__(self, constants: Constants):
        self.constants = constants
        self.ptr = lib().HPMCcreateHistoPyramid(constants.ptr)
        if not self.ptr:
            raise HPMCError(_capi.ERR_INVALID_HANDLE, "HPMCcreateHistoPyramid")
        self._keep = {}

    # -- reference setters -------------------------------------------------
    def set_lattice_size(self, x, y, z):
        lib().HPMCsetLatticeSize(self.ptr, int(x), int(y), int(z))

    def set_grid_size(self, x, y, z):
        lib().HPMCsetGridSize(self.ptr, int(x), int(y), int(z))

    def set_grid_extent(self, x, y, z):
        lib().HPMCsetGridExtent(self.ptr, float(x), float(y), float(z))

    def set_field_as_binary(self):
        lib().HPMCsetFieldAsBinary(self.ptr)

    def set_field_as_continuous(self):
        lib().HPMCsetFieldAsContinuous(self.ptr)

    def set_field_texture3d(self, name: int, gradient: bool = False):
        lib().HPMCsetFieldTexture3D(self.ptr, int(name), 1 if gradient else 0)

    def set_field_custom(self, functor: str, builder_texunit: int = 0, gradient: bool = False):
        lib().HPMCsetFieldCustom(self.ptr, functor.encode(), int(builder_texunit), 1 if gradient else 0)

    def builder_program(self) -> int:
        return int(lib().HPMCgetBuilderProgram(self.ptr))

    def build(self, iso: float):
        lib().HPMCbuildHistopyramid(self.ptr, float(iso))

    def acquire_number_of_vertices(self) -> int:
        return int(lib().HPMCacquireNumberOfVertices(self.ptr))

    # -- CUDA-native --------------------------------------------------------
    @property
    def last_error(self) -> int:
        return int(lib().HPMCgetLastError(self.ptr))

    def set_field_device(self, field, unorm: bool = False):
        """Field tensor (z, y, x) float32 or uint8, or (z, y, x, 4) float32
        (gradient + value), on the current CUDA device."""
        _field_layout(field)
        es = field.element_size()
        self._keep["field"] = field
        fz, fy, fx = field.shape[:3]
        self.set_lattice_size(fx, fy, fz)
        _check(lib().HPMCsetFieldDevice(self.ptr, field.data_ptr(), _scalar_type(field, unorm),
                                        field.stride(1) * es, field.stride(0) * es), "HPMCsetFieldDevice")

    def set_builder_uniforms(self, values):
        import array

        buf = array.array("f", [float(v) for v in values])
        addr, n = buf.buffer_info()
        self._keep["uniforms"] = buf
        _check(lib().HPMCsetBuilderUniforms(self.ptr, addr, n), "HPMCsetBuilderUniforms")

    def set_stream(self, stream):
        handle = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        _check(lib().HPMCsetStream(self.ptr, handle), "HPMCsetStream")

    def set_normal_mode(self, mode: int):
        _check(lib().HPMCsetNormalMode(self.ptr, int(mode)), "HPMCsetNormalMode")

    def set_code_capture(self, codes):
        self._keep["codes"] = codes
        _check(lib().HPMCsetCodeCapture(self.ptr, _ptr(codes)), "HPMCsetCodeCapture")

    def layout(self):
        out = (C.c_int * 6)()
        _check(lib().HPMCgetLayout(self.ptr, out), "HPMCgetLayout")
        return tuple(out)

    def read_level(self, level: int):
        import numpy as np

        l2 = self.layout()[4]
        e = l2 + 1 - level
        n = 1 if e <= 0 else 1 << (2 * e)
        out = np.zeros(n, np.uint32)
        _check(lib().HPMCreadLevel(self.ptr, int(level), out.ctypes.data, n), "HPMCreadLevel")
        return out

    def classify_path(self) -> int:
        """1: TMA column kernel, 0: generic per-block kernel (last build)."""
        p = C.c_int(-1)
        _check(lib().HPMCgetClassifyPath(self.ptr, C.byref(p)), "HPMCgetClassifyPath")
        return int(p.value)

    def device_status(self) -> int:
        s = C.c_uint(0)
        _check(lib().HPMCgetDeviceStatus(self.ptr, C.byref(s)), "HPMCgetDeviceStatus")
        return int(s.value)

    def set_test_stall(self, box: int, wait_limit_us: int = 0):
        """Failure-detection test hook (HPMCsetTestStall): classifier box `box`
        never arrives, so the build times out; box < 0 turns it off."""
        _check(lib().HPMCsetTestStall(self.ptr, int(box), int(wait_limit_us)), "HPMCsetTestStall")

    def close(self):
        if self.ptr:
            lib().HPMCdestroyHandle(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TraversalHandle:
    """HPMCcreateTraversalHandle and extraction (hpmc.h:478-544)."""

    def __init__(self, hp: HistoPyramid):
        self.hp = hp
        self.ptr = lib().HPMCcreateTraversalHandle(hp.ptr)
        if not self.ptr:
            raise HPMCError(hp.last_error or _capi.ERR_LAYOUT, "HPMCcreateTraversalHandle")
        self._keep = {}

    def set_buffers(self, pos, nrm, capacity: int | None = None):
        cap = capacity if capacity is not None else (pos if pos is not None else nrm).shape[0]
        self._keep["buf"] = (pos, nrm)
        _check(lib().HPMCsetTraversalHandleBuffers(self.ptr, _ptr(pos), _ptr(nrm), int(cap)),
               "HPMCsetTraversalHandleBuffers")

    def set_feedback_buffer(self, buf, capacity: int | None = None):
        cap = capacity if capacity is not None else buf.numel() // 6
        self._keep["fb"] = buf
        _check(lib().HPMCsetTraversalHandleFeedbackBuffer(self.ptr, _ptr(buf), int(cap)),
               "HPMCsetTraversalHandleFeedbackBuffer")

    def set_debug_buffers(self, cell_info=None, t=None):
        self._keep["dbg"] = (cell_info, t)
        _check(lib().HPMCsetTraversalDebugBuffers(self.ptr, _ptr(cell_info), _ptr(t)),
               "HPMCsetTraversalDebugBuffers")

    def extract(self) -> bool:
        return bool(lib().HPMCextractVertices(self.ptr))

    def extract_feedback(self) -> bool:
        return bool(lib().HPMCextractVerticesTransformFeedback(self.ptr))

    def extract_to(self, pos, nrm, capacity: int | None = None, sync: bool = True) -> int:
        cap = capacity if capacity is not None else (pos if pos is not None else nrm).shape[0]
        n = C.c_uint64(0)
        st = lib().HPMCextractVerticesToBuffers(self.ptr, _ptr(pos), _ptr(nrm), int(cap),
                                                C.byref(n) if sync else None)
        if st not in (_capi.OK, _capi.ERR_CAPACITY):
            raise HPMCError(st, "HPMCextractVerticesToBuffers")
        return int(n.value)

    def extract_indexed(self, pos, nrm, indices, vertex_capacity: int | None = None,
                        index_capacity: int | None = None):
        """Welded output (HPMCextractVerticesIndexed): one vertex per crossed
        edge in first-occurrence order, one index per soup vertex.  Returns
        (unique vertices, indices); raises unless both fit."""
        vcap = vertex_capacity if vertex_capacity is not None else (pos if pos is not None else nrm).shape[0]
        icap = index_capacity if index_capacity is not None else indices.numel()
        nv, ni = C.c_uint64(0), C.c_uint64(0)
        _check(lib().HPMCextractVerticesIndexed(self.ptr, _ptr(pos), _ptr(nrm), int(vcap), _ptr(indices), int(icap),
                                                C.byref(nv), C.byref(ni)), "HPMCextractVerticesIndexed")
        return int(nv.value), int(ni.value)

    def adjoint(self, dpos, dnrm, count: int, dfield):
        _check(lib().HPMCextractVerticesAdjoint(self.ptr, _ptr(dpos), _ptr(dnrm), int(count),
                                                dfield.data_ptr()), "HPMCextractVerticesAdjoint")

    def close(self):
        if self.ptr:
            lib().HPMCdestroyTraversalHandle(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Batched extraction (HPMCcreateBatch ... HPMCbatchExtract): many (z, y, x)
    CUDA fields of one dtype, uneven sizes and per-volume iso-values, extracted by
    one CUDA-graph replay.  Volume v's vertices are rows offsets[v]:offsets[v+1]."""

    def __init__(self, fields, isos, *, extents=None, normals: int = NORMALS_FORWARD, unorm: bool = False,
                 constants: Constants | None = None):
        self.constants = constants or default_constants()
        self.fields = list(fields)
        n = len(self.fields)
        vols = (_capi.BatchVolume * n)()
        for i, (f, iso) in enumerate(zip(self.fields, isos)):
            if not f.is_cuda or f.stride(2) != 1:
                raise ValueError("fields must be CUDA tensors with unit stride along x")
            es = f.element_size()
            fz, fy, fx = f.shape
            vols[i].field = f.data_ptr()
            vols[i].scalar_type = _scalar_type(f, unorm)
            vols[i].size[:] = [fx, fy, fz]
            vols[i].row_pitch_bytes = f.stride(1) * es
            vols[i].slice_pitch_bytes = f.stride(0) * es
            vols[i].iso = float(iso)
            ext = extents[i] if extents is not None else (1.0, 1.0, 1.0)
            vols[i].extent[:] = [float(e) for e in ext]
        self.count = n
        self.ptr = C.c_void_p()
        _check(lib().HPMCcreateBatch(self.constants.ptr, C.cast(vols, C.c_void_p), n, C.byref(self.ptr)),
               "HPMCcreateBatch")
        self.set_normal_mode(normals)

    def set_normal_mode(self, mode: int):
        _check(lib().HPMCbatchSetNormalMode(self.ptr, int(mode)), "HPMCbatchSetNormalMode")

    def set_iso_values(self, isos):
        buf = (C.c_float * self.count)(*[float(v) for v in isos])
        _check(lib().HPMCbatchSetIsoValues(self.ptr, buf), "HPMCbatchSetIsoValues")

    def set_tuning(self, column_slices: int = 0, traverse_ctas_per_sm: int = 0, rounds: int = 0):
        _check(lib().HPMCbatchSetTuning(self.ptr, column_slices, traverse_ctas_per_sm, rounds), "HPMCbatchSetTuning")

    def tuning(self):
        out = (C.c_int * 3)()
        _check(lib().HPMCbatchGetTuning(self.ptr, out), "HPMCbatchGetTuning")
        return tuple(out)

    def extract(self, pos, nrm, capacity: int | None = None, stream=None):
        """Asynchronous: build, count and extract every volume into pos/nrm (float4 rows)."""
        import torch

        cap = capacity if capacity is not None else (pos if pos is not None else nrm).shape[0]
        st = stream if stream is not None else torch.cuda.current_stream()
        _check(lib().HPMCbatchExtract(self.ptr, _ptr(pos), _ptr(nrm), int(cap), st.cuda_stream), "HPMCbatchExtract")

    def offsets(self, allow_truncation: bool = False):
        """count + 1 output offsets of the last extraction (waits for it)."""
        out = (C.c_ulonglong * (self.count + 1))()
        st = lib().HPMCbatchGetOffsets(self.ptr, out)
        if st != _capi.OK and not (allow_truncation and st == _capi.ERR_CAPACITY):
            raise HPMCError(st, "HPMCbatchGetOffsets")
        return [int(v) for v in out]

    def set_test_stall(self, volume: int, box: int, wait_limit_us: int = 0):
        """Failure-detection test hook (HPMCbatchSetTestStall)."""
        _check(lib().HPMCbatchSetTestStall(self.ptr, int(volume), int(box), int(wait_limit_us)),
               "HPMCbatchSetTestStall")

    def autotune(self, pos, nrm, capacity: int | None = None, stream=None):
        import torch

        cap = capacity if capacity is not None else (pos if pos is not None else nrm).shape[0]
        st = stream if stream is not None else torch.cuda.current_stream()
        out = (C.c_int * 3)()
        _check(lib().HPMCbatchAutotune(self.ptr, _ptr(pos), _ptr(nrm), int(cap), st.cuda_stream, out),
               "HPMCbatchAutotune")
        return tuple(out)

    def close(self):
        if self.ptr:
            lib().HPMCdestroyBatch(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_constants = None


def default_constants() -> Constants:
    global _default_constants
    if _default_constants is None:
        _default_constants = Constants()
    return _default_constants


def extract(field, iso: float, *, cells=None, extent=(1.0, 1.0, 1.0), normals: int = NORMALS_FORWARD,
            binary: bool = False, unorm: bool = False, debug: bool = False):
    """One-shot extraction of a (z, y, x) CUDA field: returns (pos, nrm[, info, t]),
    float4 per vertex, in the reference's vertex order."""
    import torch

    hp = HistoPyramid(default_constants())
    hp.set_stream(torch.cuda.current_stream())
    hp.set_field_device(field, unorm=unorm)
    if cells is not None:
        hp.set_grid_size(*cells)
    hp.set_grid_extent(*extent)
    if binary:
        hp.set_field_as_binary()
    hp.set_normal_mode(normals)
    hp.build(iso)
    n = hp.acquire_number_of_vertices()
    if hp.last_error:
        raise HPMCError(hp.last_error, "build")
    th = TraversalHandle(hp)
    pos = torch.empty((max(n, 1), 4), dtype=torch.float32, device=field.device)
    nrm = torch.empty_like(pos)
    info = t = None
    if debug:
        info = torch.empty((max(n, 1), 4), dtype=torch.int32, device=field.device)
        t = torch.empty((max(n, 1),), dtype=torch.float32, device=field.device)
        th.set_debug_buffers(info, t)
    written = th.extract_to(pos, nrm, n)
    th.close()
    hp.close()
    if debug:
        return pos[:written], nrm[:written], info[:written], t[:written]
    return pos[:written], nrm[:written]
