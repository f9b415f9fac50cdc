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


def _static_path(hpmc, field, iso, normals, capacity, *, outputs=True, status_out=None):
    """HPMCextractStatic through the C ABI; `field` may be a strided view
    (unit stride along x).  Returns (full count, (positions, normals))."""
    import torch

    from hpmc_b200 import _capi

    L = hpmc.lib()
    fz, fy, fx = field.shape
    es = field.element_size()
    pos = torch.full((max(capacity, 1), 4), float("nan"), dtype=torch.float32, device=field.device)
    nrm = torch.full_like(pos, float("nan"))
    count = torch.zeros(1, dtype=torch.int32, device=field.device)
    status = torch.full((1,), -1, dtype=torch.int32, device=field.device)
    stype = _capi.SCALAR_F32 if field.dtype == torch.float32 else _capi.SCALAR_U8
    st = L.HPMCextractStatic(field.data_ptr(), stype, fx, fy, fz, field.stride(1) * es, field.stride(0) * es,
                             float(iso), int(normals), None, pos.data_ptr() if outputs else None,
                             nrm.data_ptr() if outputs else None, capacity, count.data_ptr(), status.data_ptr(),
                             C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _capi.OK, st
    torch.cuda.synchronize()
    n = int(count.item())
    if status_out is not None:
        status_out.append(int(status.item()))
    m = min(n, capacity)
    return n, (pos[:m].cpu().numpy(), nrm[:m].cpu().numpy())


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


def test_static_edge_cases_match_allocating_path(hpmc, oracle):
    """Documented behaviours: the generic classifier for lattices too narrow
    for the column path, a pitched (not 16-byte aligned) field, truncation
    (the full count is reported, the prefix is written, status bit 2), NULL
    outputs, and a small call after a large one (state left in the scratch
    by the larger call must not leak)."""
    import torch

    from hpmc_b200 import datasets
    from tests.gpu_helpers import oracle_expect

    rng = np.random.default_rng(5)
    cases = []
    small = rng.normal(size=(30, 40, 12)).astype(np.float32)  # tiles narrower than 32 cells: generic path
    cases.append(("narrow", torch.from_numpy(small).cuda(), small, 0.0))
    big = torch.zeros((33, 50, 64 + 3), dtype=torch.float32, device="cuda")
    pitched_np = rng.normal(size=(33, 50, 64)).astype(np.float32)
    big[:, :, :64] = torch.from_numpy(pitched_np).cuda()
    cases.append(("pitched", big[:, :, :64], pitched_np, 0.0))
    large_np, iso_l = datasets.cayley(150)
    cases.append(("large", torch.from_numpy(large_np).cuda(), large_np, iso_l))
    tiny = rng.normal(size=(9, 8, 10)).astype(np.float32)
    cases.append(("small-after-large", torch.from_numpy(tiny).cuda(), tiny, 0.0))
    for name, field, field_np, iso in cases:
        for normals in (0, 1):
            n_ref, (p_ref, q_ref) = _handle_path(hpmc, field, iso, normals)
            st = []
            n, (p, q) = _static_path(hpmc, field, iso, normals, capacity=n_ref + 8, status_out=st)
            assert n == n_ref and st == [0], (name, n, n_ref, st)
            np.testing.assert_allclose(p, p_ref, rtol=0, atol=1e-6)
            np.testing.assert_allclose(q, q_ref, rtol=0, atol=1e-6)
        # against the oracle as well (positions within the parity tolerance)
        e = oracle_expect(oracle, field_np, iso, normals=1)
        assert n == e["total"], name
        spacing = 1.0 / np.array(e["L"].cells, np.float64)
        dp = np.abs(p[:, :3].astype(np.float64) - e["pos"])
        assert (dp <= 1e-5 * spacing[None, :] + 4 * np.finfo(np.float32).eps * np.abs(e["pos"])).all(), name
        # truncation: the full count, the written prefix, the capacity bit
        half = n_ref // 2
        st = []
        n2, (p2, _) = _static_path(hpmc, field, iso, 1, capacity=half, status_out=st)
        assert n2 == n_ref and st == [2], (name, n2, st)
        np.testing.assert_allclose(p2, p[:half], rtol=0, atol=1e-6)
        # NULL outputs: the count alone
        n3, _ = _static_path(hpmc, field, iso, 1, capacity=0, outputs=False)
        assert n3 == n_ref


def test_static_rejects_lattices_beyond_scratch(hpmc):
    import torch

    from hpmc_b200 import _capi

    field = torch.zeros((256, 256, 256), dtype=torch.uint8, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = hpmc.lib().HPMCextractStatic(field.data_ptr(), _capi.SCALAR_U8, 256, 256, 256, 0, 0, 128.0, 0, None,
                                      None, None, 0, count.data_ptr(), None, None)
    assert st == _capi.ERR_TOO_LARGE
