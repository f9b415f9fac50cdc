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


def test_no_cpu_fallback_without_library(monkeypatch, tmp_path):
    """The product raises when its CUDA library is missing."""
    import hpmc_b200._capi as capi

    monkeypatch.setattr(capi, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(capi, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        capi.lib()
