"""HPMCextractStatic: extraction for callers that cannot allocate device memory.

Render engines and plugins that are handed a fixed GPU memory budget, and
real-time loops where cudaMalloc/cudaFree (which synchronise the device) are
not allowed, use this entry point: all of its scratch lives in one fixed
device array inside the library.  These tests call it through the C ABI and
check its output against the allocating entry points (HPMCbuildHistopyramid +
HPMCextractVerticesToBuffers) on two calls in a row, so the second call also
shows that state left in the shared scratch by the first does not leak.

The file name sorts last so that a run that stops at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _handle_path(hpmc, field, iso, normals):
    """Reference result through the allocating C-ABI entry points."""
    import torch

    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(torch.cuda.current_stream())
    hp.set_field_device(field)
    hp.set_normal_mode(normals)
    hp.build(iso)
    n = hp.acquire_number_of_vertices()
    th = hpmc.TraversalHandle(hp)
    pos = torch.zeros((max(n, 1), 4), dtype=torch.float32, device=field.device)
    nrm = torch.zeros_like(pos)
    th.extract_to(pos, nrm, n)
    torch.cuda.synchronize()
    out = pos[:n].cpu().numpy(), nrm[:n].cpu().numpy()
    th.close()
    hp.close()
    return n, out


def _static_path(hpmc, field, iso, normals, capacity):
    import torch

    from hpmc_b200 import _capi

    L = hpmc.lib()
    fz, fy, fx = field.shape
    pos = torch.full((capacity, 4), float("nan"), dtype=torch.float32, device=field.device)
    nrm = torch.full_like(pos, float("nan"))
    count = torch.zeros(1, dtype=torch.int32, device=field.device)
    stype = _capi.SCALAR_F32 if field.dtype == torch.float32 else _capi.SCALAR_U8
    st = L.HPMCextractStatic(field.data_ptr(), stype, fx, fy, fz, 0, 0, float(iso), int(normals), None,
                             pos.data_ptr(), nrm.data_ptr(), capacity, count.data_ptr(),
                             C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _capi.OK, st
    torch.cuda.synchronize()
    n = int(count.item())
    return n, (pos[:n].cpu().numpy(), nrm[:n].cpu().numpy())


def _fields():
    from hpmc_b200 import datasets

    a, iso_a = datasets.metaballs_64()
    rng = np.random.default_rng(17)
    b = rng.integers(100, 156, size=(40, 72, 96)).astype(np.uint8)  # ties at 128
    return [(a, iso_a, 1), (b, 128.0, 0)]


def test_static_matches_allocating_path_twice(hpmc):
    """Two calls in a row, each equal to the allocating entry points."""
    import torch

    for field_np, iso, normals in _fields():
        field = torch.from_numpy(field_np).cuda()
        n_ref, (p_ref, n_ref_arr) = _handle_path(hpmc, field, iso, normals)
        n, (p, nn) = _static_path(hpmc, field, iso, normals, capacity=n_ref + 16)
        assert n == n_ref and n > 0
        # same kernels on the same inputs: within the parity tolerance (equal in practice)
        np.testing.assert_allclose(p, p_ref, rtol=0, atol=1e-6)
        np.testing.assert_allclose(nn, n_ref_arr, rtol=0, atol=1e-6)


def test_static_rejects_lattices_beyond_scratch(hpmc):
    import torch

    from hpmc_b200 import _capi

    field = torch.zeros((256, 256, 256), dtype=torch.uint8, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = hpmc.lib().HPMCextractStatic(field.data_ptr(), _capi.SCALAR_U8, 256, 256, 256, 0, 0, 128.0, 0, None,
                                      None, None, 0, count.data_ptr(), None)
    assert st == _capi.ERR_TOO_LARGE
