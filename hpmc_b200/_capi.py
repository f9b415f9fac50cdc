"""ctypes binding of ``libhpmc_b200.so`` (the C ABI declared in include/hpmc.h).

The library is the product: every call below goes straight to the compiled
sm_100a code.  There is no Python or CPU fallback; if the library is missing
this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "_lib", "libhpmc_b200.so")
HEADER = os.path.join(os.path.dirname(_PKG), "include", "hpmc.h")

# HPMCStatus
OK = 0
ERR_INVALID_HANDLE = 1
ERR_INVALID_VALUE = 2
ERR_LAYOUT = 3
ERR_UNSUPPORTED = 4
ERR_CUDA = 5
ERR_OUT_OF_MEMORY = 6
ERR_CAPACITY = 7
ERR_NOT_BUILT = 8
ERR_BROKEN = 9
ERR_NO_FIELD = 10
ERR_OVERFLOW = 11
ERR_TIMEOUT = 12
ERR_TOO_LARGE = 13
STATIC_SCRATCH_BYTES = 16 << 20

STATUS_NAMES = {v: k for k, v in globals().items() if k.startswith("ERR_") or k == "OK"}

# HPMCScalarType
SCALAR_F32, SCALAR_U8, SCALAR_UNORM8, SCALAR_F32X4 = 0, 1, 2, 3
# HPMCNormalMode
NORMALS_FORWARD, NORMALS_CENTRAL = 0, 1

vp = C.c_void_p
_SIGS = {
    # reference entry points (hpmc/include/hpmc.h:310-544)
    "HPMCcreateConstants": (vp, [C.c_int, C.c_int]),
    "HPMCdestroyConstants": (None, [vp]),
    "HPMCcreateHistoPyramid": (vp, [vp]),
    "HPMCsetLatticeSize": (None, [vp, C.c_int, C.c_int, C.c_int]),
    "HPMCsetFieldAsBinary": (None, [vp]),
    "HPMCsetFieldAsContinuous": (None, [vp]),
    "HPMCsetGridSize": (None, [vp, C.c_int, C.c_int, C.c_int]),
    "HPMCsetGridExtent": (None, [vp, C.c_float, C.c_float, C.c_float]),
    "HPMCsetFieldTexture3D": (None, [vp, C.c_uint, C.c_ubyte]),
    "HPMCsetFieldCustom": (None, [vp, C.c_char_p, C.c_uint, C.c_ubyte]),
    "HPMCgetBuilderProgram": (C.c_uint, [vp]),
    "HPMCdestroyHandle": (None, [vp]),
    "HPMCbuildHistopyramid": (None, [vp, C.c_float]),
    "HPMCacquireNumberOfVertices": (C.c_uint, [vp]),
    "HPMCcreateTraversalHandle": (vp, [vp]),
    "HPMCdestroyTraversalHandle": (None, [vp]),
    "HPMCgetTraversalShaderFunctions": (vp, [vp]),
    "HPMCsetTraversalHandleProgram": (C.c_bool, [vp, C.c_uint, C.c_uint, C.c_uint, C.c_uint]),
    "HPMCextractVertices": (C.c_bool, [vp]),
    "HPMCextractVerticesTransformFeedback": (C.c_bool, [vp]),
    "HPMCextractVerticesTransformFeedbackNV": (C.c_bool, [vp]),
    "HPMCextractVerticesTransformFeedbackEXT": (C.c_bool, [vp]),
    # CUDA-native entry points
    "HPMCgetLastError": (C.c_int, [vp]),
    "HPMCregisterDeviceField": (C.c_uint, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_size_t, C.c_size_t]),
    "HPMCunregisterDeviceField": (None, [C.c_uint]),
    "HPMCsetFieldDevice": (C.c_int, [vp, vp, C.c_int, C.c_size_t, C.c_size_t]),
    "HPMCsetBuilderUniforms": (C.c_int, [vp, vp, C.c_int]),
    "HPMCsetStream": (C.c_int, [vp, vp]),
    "HPMCsetNormalMode": (C.c_int, [vp, C.c_int]),
    "HPMCgetDeviceVertexCount": (C.c_int, [vp, C.POINTER(vp)]),
    "HPMCsetTraversalHandleBuffers": (C.c_int, [vp, vp, vp, C.c_size_t]),
    "HPMCsetTraversalHandleFeedbackBuffer": (C.c_int, [vp, vp, C.c_size_t]),
    "HPMCextractVerticesToBuffers": (C.c_int, [vp, vp, vp, C.c_size_t, C.POINTER(C.c_uint64)]),
    "HPMCextractVerticesAdjoint": (C.c_int, [vp, vp, vp, C.c_uint64, vp]),
    "HPMCsetCodeCapture": (C.c_int, [vp, vp]),
    "HPMCgetLayout": (C.c_int, [vp, C.POINTER(C.c_int)]),
    "HPMCreadLevel": (C.c_int, [vp, C.c_int, vp, C.c_size_t]),
    "HPMCsetTraversalDebugBuffers": (C.c_int, [vp, vp, vp]),
    "HPMCgetDeviceStatus": (C.c_int, [vp, C.POINTER(C.c_uint)]),
    "HPMCgetClassifyPath": (C.c_int, [vp, C.POINTER(C.c_int)]),
    "HPMCsetTestStall": (C.c_int, [vp, C.c_int, C.c_uint]),
    "HPMCregisterFieldFunctor": (C.c_int, [C.c_char_p, vp]),
    "HPMCunregisterFieldFunctor": (C.c_int, [C.c_char_p]),
    "HPMCextractStatic": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_size_t, C.c_size_t, C.c_float,
                                    C.c_int, C.POINTER(C.c_float), vp, vp, C.c_size_t, vp, vp, vp]),
    "HPMCextractVerticesIndexed": (C.c_int, [vp, vp, vp, C.c_size_t, vp, C.c_size_t, C.POINTER(C.c_uint64),
                                             C.POINTER(C.c_uint64)]),
    # batched extraction
    "HPMCcreateBatch": (C.c_int, [vp, vp, C.c_int, C.POINTER(vp)]),
    "HPMCdestroyBatch": (None, [vp]),
    "HPMCbatchSetIsoValues": (C.c_int, [vp, C.POINTER(C.c_float)]),
    "HPMCbatchSetNormalMode": (C.c_int, [vp, C.c_int]),
    "HPMCbatchExtract": (C.c_int, [vp, vp, vp, C.c_size_t, vp]),
    "HPMCbatchGetOffsets": (C.c_int, [vp, C.POINTER(C.c_ulonglong)]),
    "HPMCbatchGetDeviceOffsets": (C.c_int, [vp, C.POINTER(vp)]),
    "HPMCbatchSetTuning": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
    "HPMCbatchGetTuning": (C.c_int, [vp, C.POINTER(C.c_int)]),
    "HPMCbatchAutotune": (C.c_int, [vp, vp, vp, C.c_size_t, vp, C.POINTER(C.c_int)]),
    "HPMCbatchSetTestStall": (C.c_int, [vp, C.c_int, C.c_int, C.c_uint]),
}


class BatchVolume(C.Structure):
    """HPMCBatchVolume (include/hpmc.h)."""

    _fields_ = [
        ("field", C.c_void_p),
        ("scalar_type", C.c_int),
        ("size", C.c_int * 3),
        ("row_pitch_bytes", C.c_size_t),
        ("slice_pitch_bytes", C.c_size_t),
        ("iso", C.c_float),
        ("extent", C.c_float * 3),
    ]

_lib = None


def lib() -> C.CDLL:
    """Load the extension library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"hpmc_b200 CUDA library missing: {LIB_PATH}. Build it with "
                "`python -m hpmc_b200.build` (there is no CPU fallback).")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols() -> list[str]:
    """Entry points declared by include/hpmc.h (for the export check)."""
    with open(HEADER) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(HPMC[A-Za-z0-9]+)\s*\(", text)))
