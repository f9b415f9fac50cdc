"""The C-ABI library: it loads, exports every entry point include/hpmc.h
declares, and honours the reference's NULL-handle conventions.  No compute
calls (CPU only)."""
from __future__ import annotations

import ctypes as C
import subprocess

import pytest


def test_library_exports_every_declared_symbol(hpmc):
    from hpmc_b200 import _capi

    declared = _capi.declared_symbols()
    assert len(declared) >= 38
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    # every declared symbol is bound in the ctypes table too
    assert set(declared) <= set(_capi._SIGS)


def test_reference_entry_points_present(hpmc):
    """All 22 functions of the reference's public header (hpmc/include/hpmc.h:310-544)."""
    ref_api = [
        "HPMCcreateConstants", "HPMCdestroyConstants", "HPMCcreateHistoPyramid", "HPMCsetLatticeSize",
        "HPMCsetFieldAsBinary", "HPMCsetFieldAsContinuous", "HPMCsetGridSize", "HPMCsetGridExtent",
        "HPMCsetFieldTexture3D", "HPMCsetFieldCustom", "HPMCgetBuilderProgram", "HPMCdestroyHandle",
        "HPMCbuildHistopyramid", "HPMCacquireNumberOfVertices", "HPMCcreateTraversalHandle",
        "HPMCdestroyTraversalHandle", "HPMCgetTraversalShaderFunctions", "HPMCsetTraversalHandleProgram",
        "HPMCextractVertices", "HPMCextractVerticesTransformFeedback",
        "HPMCextractVerticesTransformFeedbackNV", "HPMCextractVerticesTransformFeedbackEXT",
    ]
    L = hpmc.lib()
    for name in ref_api:
        assert hasattr(L, name), name


def test_null_handle_conventions(hpmc):
    L = hpmc.lib()
    from hpmc_b200 import _capi

    assert L.HPMCcreateConstants(1, 5) is None  # GL < 2.0 rejected (constants.cpp:115-123)
    assert L.HPMCcreateHistoPyramid(None) is None
    assert L.HPMCcreateTraversalHandle(None) is None
    assert L.HPMCacquireNumberOfVertices(None) == 0
    assert L.HPMCgetBuilderProgram(None) == 0
    assert L.HPMCextractVertices(None) is False
    assert L.HPMCextractVerticesTransformFeedback(None) is False
    assert L.HPMCsetTraversalHandleProgram(None, 1, 0, 1, 2) is False
    assert L.HPMCgetTraversalShaderFunctions(None) is None
    assert L.HPMCgetLastError(None) == _capi.ERR_INVALID_HANDLE
    assert L.HPMCsetStream(None, None) == _capi.ERR_INVALID_HANDLE
    assert L.HPMCsetNormalMode(None, 0) == _capi.ERR_INVALID_HANDLE
    assert L.HPMCextractVerticesAdjoint(None, None, None, 0, None) == _capi.ERR_INVALID_HANDLE
    # NULL-safe destroyers
    L.HPMCdestroyConstants(None)
    L.HPMCdestroyHandle(None)
    L.HPMCdestroyTraversalHandle(None)
    # field registry: bad arguments give name 0
    assert L.HPMCregisterDeviceField(None, 0, 4, 4, 4, 0, 0) == 0
    assert L.HPMCregisterDeviceField(C.c_void_p(16), 7, 4, 4, 4, 0, 0) == 0
    name = L.HPMCregisterDeviceField(C.c_void_p(16), 0, 4, 4, 4, 0, 0)
    assert name != 0
    L.HPMCunregisterDeviceField(name)


class _FunctorOps(C.Structure):
    """HPMCFieldFunctorOps (include/hpmc.h)."""

    _fields_ = [("abi", C.c_uint), ("volume_bytes", C.c_int), ("outputs_bytes", C.c_int),
                ("has_gradient", C.c_int), ("classify", C.c_void_p), ("traverse", C.c_void_p)]


def test_functor_registration_rules(hpmc):
    """HPMCregisterFieldFunctor checks the table before it keeps it: reserved
    and empty names, NULL tables, a wrong ABI version, descriptor sizes or
    missing launchers are refused (no CUDA call is made)."""
    from hpmc_b200 import _capi

    L = hpmc.lib()
    dummy = C.cast(C.pointer(C.c_int(0)), C.c_void_p)  # never called: only checked for NULL
    bad = [_FunctorOps(1, 0, 0, 0, dummy, dummy), _FunctorOps(99, 1, 1, 0, dummy, dummy),
           _FunctorOps(1, 1, 1, 0, None, dummy)]
    for ops in bad:
        assert L.HPMCregisterFieldFunctor(b"app:x", C.byref(ops)) == _capi.ERR_INVALID_VALUE
    assert L.HPMCregisterFieldFunctor(b"app:x", None) == _capi.ERR_INVALID_VALUE
    assert L.HPMCregisterFieldFunctor(b"hpmc:cayley", None) == _capi.ERR_INVALID_VALUE
    assert L.HPMCregisterFieldFunctor(b"", None) == _capi.ERR_INVALID_VALUE
    assert L.HPMCunregisterFieldFunctor(b"app:never-registered") == _capi.ERR_INVALID_VALUE


def test_no_cpu_fallback_without_library(monkeypatch, tmp_path):
    """The product raises when its CUDA library is missing."""
    import hpmc_b200._capi as capi

    monkeypatch.setattr(capi, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(capi, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        capi.lib()
