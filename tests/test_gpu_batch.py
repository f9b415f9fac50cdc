"""Batched extraction (HPMCcreateBatch / HPMCbatchExtract) through the C ABI.

Per volume, the batch must produce exactly what the handle path
(HPMCbuildHistopyramid + HPMCextractVerticesToBuffers) produces on that
volume -- same count, same vertex order, geometry within 1e-6 -- and the
handle path is itself pinned to the oracle (test_gpu_parity.py).  Small
volumes are also checked against the oracle directly.
"""
from __future__ import annotations

import numpy as np
import pytest

from tests.gpu_helpers import compare, oracle_expect, run_gpu

pytestmark = pytest.mark.gpu


def _metaballs(shape, seed, m):
    from hpmc_b200 import datasets

    rng = np.random.default_rng(seed)
    c = rng.uniform(0.2, 0.8, size=(m, 3))
    r = rng.uniform(0.05, 0.15, size=m)
    fz, fy, fx = shape
    return datasets.metaballs(0, c, r, shape=(fx, fy, fz))


# (z, y, x): cubes of uneven edges, non-cubic volumes, a volume too narrow
# for the column classifier (per-volume generic launch) and a one-block pyramid
SHAPES = [(32, 32, 32), (36, 36, 36), (52, 52, 52), (100, 100, 100), (40, 48, 64), (20, 20, 20), (12, 12, 12),
          (9, 17, 33), (64, 64, 64), (33, 97, 36)]


def _volumes(dtype="f32"):
    vols = []
    for i, s in enumerate(SHAPES):
        f = _metaballs(s, 100 + i, 4 + 3 * i)
        iso = 0.8 + 0.07 * i
        if dtype == "u8":
            f = np.clip(np.rint(f * 60.0), 0, 255).astype(np.uint8)
            iso = float(round(iso * 60.0))  # samples equal to iso: ties
        vols.append((f, iso))
    return vols


def _batch_run(hpmc, tensors, isos, normals, capacity=None, tuning=None):
    import torch

    b = hpmc.Batch(tensors, isos, normals=normals)
    if tuning is not None:
        b.set_tuning(*tuning)
    cap = capacity
    if cap is None:
        # first pass to size the outputs
        tmp = torch.empty((1, 4), dtype=torch.float32, device="cuda")
        b.extract(tmp, tmp, 0)
        cap = b.offsets(allow_truncation=True)[-1]
    pos = torch.full((max(cap, 1), 4), float("nan"), dtype=torch.float32, device="cuda")
    nrm = torch.full_like(pos, float("nan"))
    b.extract(pos, nrm, cap)
    offs = b.offsets(allow_truncation=capacity is not None)
    torch.cuda.synchronize()
    return b, offs, pos.cpu().numpy(), nrm.cpu().numpy()


@pytest.mark.parametrize("normals", [0, 1])
@pytest.mark.parametrize("dtype", ["f32", "u8"])
def test_batch_equals_handle_path(hpmc, dtype, normals):
    import torch

    vols = _volumes(dtype)
    tensors = [torch.from_numpy(f).cuda() for f, _ in vols]
    b, offs, pos, nrm = _batch_run(hpmc, tensors, [iso for _, iso in vols], normals)
    assert offs[0] == 0 and all(offs[i] <= offs[i + 1] for i in range(len(vols)))
    for i, (f, iso) in enumerate(vols):
        g = run_gpu(hpmc, f, iso, normals=normals, capture_codes=False)
        lo, hi = offs[i], offs[i + 1]
        assert hi - lo == g["n"], (i, hi - lo, g["n"])
        np.testing.assert_allclose(pos[lo:hi], g["pos"], rtol=0, atol=1e-6)
        np.testing.assert_allclose(nrm[lo:hi], g["nrm"], rtol=0, atol=1e-6)
    b.close()


def test_batch_small_volumes_vs_oracle(hpmc, oracle):
    import torch

    vols = _volumes("f32")[:3] + [_volumes("f32")[6]]
    tensors = [torch.from_numpy(f).cuda() for f, _ in vols]
    b, offs, pos, nrm = _batch_run(hpmc, tensors, [iso for _, iso in vols], 1)
    for i, (f, iso) in enumerate(vols):
        e = oracle_expect(oracle, f, iso, normals=1)
        lo, hi = offs[i], offs[i + 1]
        assert hi - lo == e["total"]
        spacing = 1.0 / (np.array(f.shape[::-1], np.float64) - 1.0)
        dp = np.abs(pos[lo:hi, :3].astype(np.float64) - e["pos"])
        assert (dp <= 1e-5 * spacing[None, :] + 4 * np.finfo(np.float32).eps * np.abs(e["pos"])).all()
    b.close()


def test_batch_capacity_truncation(hpmc):
    import torch

    vols = _volumes("f32")
    tensors = [torch.from_numpy(f).cuda() for f, _ in vols]
    isos = [iso for _, iso in vols]
    b, offs, pos, nrm = _batch_run(hpmc, tensors, isos, 0)
    total = offs[-1]
    cap = total // 2 + 3
    b2, offs2, pos2, nrm2 = _batch_run(hpmc, tensors, isos, 0, capacity=cap)
    assert offs2 == offs  # offsets describe the full result
    np.testing.assert_array_equal(pos2[:cap], pos[:cap])
    assert np.isnan(pos2[cap:]).all() if pos2.shape[0] > cap else True
    b.close()
    b2.close()


def test_batch_iso_update_and_replay(hpmc):
    import torch

    vols = _volumes("f32")[:5]
    tensors = [torch.from_numpy(f).cuda() for f, _ in vols]
    b, offs, _, _ = _batch_run(hpmc, tensors, [iso for _, iso in vols], 0)
    new_isos = [1.3 - 0.05 * i for i in range(len(vols))]
    b.set_iso_values(new_isos)
    cap = 4 * offs[-1] + 1024
    pos = torch.zeros((cap, 4), dtype=torch.float32, device="cuda")
    nrm = torch.zeros_like(pos)
    for _ in range(2):  # the second call replays the captured graph
        b.extract(pos, nrm, cap)
        offs2 = b.offsets()
    p = pos.cpu().numpy()
    for i, (f, _) in enumerate(vols):
        g = run_gpu(hpmc, f, new_isos[i], capture_codes=False)
        assert offs2[i + 1] - offs2[i] == g["n"]
        np.testing.assert_allclose(p[offs2[i]:offs2[i + 1]], g["pos"], rtol=0, atol=1e-6)
    b.close()


def test_batch_autotune_keeps_results(hpmc):
    import torch

    vols = _volumes("f32")
    tensors = [torch.from_numpy(f).cuda() for f, _ in vols]
    b, offs, pos, nrm = _batch_run(hpmc, tensors, [iso for _, iso in vols], 1)
    cap = offs[-1]
    p2 = torch.zeros((cap, 4), dtype=torch.float32, device="cuda")
    n2 = torch.zeros_like(p2)
    chosen = b.autotune(p2, n2, cap)
    assert chosen[0] in (7, 15, 31, 63) and chosen[1] in (2, 3, 4) and chosen[2] in (4, 8, 16, 32, 64)
    assert b.tuning() == chosen
    p2.zero_()
    b.extract(p2, n2, cap)
    assert b.offsets() == offs
    np.testing.assert_allclose(p2.cpu().numpy(), pos, rtol=0, atol=1e-6)
    np.testing.assert_allclose(n2.cpu().numpy(), nrm, rtol=0, atol=1e-6)
    b.close()


@pytest.mark.parametrize("tuning", [(7, 2, 4), (63, 4, 16), (15, 3, 8)])
def test_batch_tuning_choices_agree(hpmc, tuning):
    import torch

    vols = _volumes("f32")
    tensors = [torch.from_numpy(f).cuda() for f, _ in vols]
    isos = [iso for _, iso in vols]
    b0, offs0, pos0, _ = _batch_run(hpmc, tensors, isos, 0)
    b1, offs1, pos1, _ = _batch_run(hpmc, tensors, isos, 0, tuning=tuning)
    assert offs0 == offs1
    np.testing.assert_allclose(pos1, pos0, rtol=0, atol=1e-6)
    b0.close()
    b1.close()


def test_batch_rejects_mixed_types(hpmc):
    import torch

    a = torch.zeros((8, 8, 8), dtype=torch.float32, device="cuda")
    u = torch.zeros((8, 8, 8), dtype=torch.uint8, device="cuda")
    with pytest.raises(hpmc.HPMCError):
        hpmc.Batch([a, u], [0.5, 0.5])


@pytest.mark.slow
def test_batch_64_uneven_volumes(hpmc):
    """The 64-volume batch workload: every volume's count and vertices equal
    the handle path's."""
    import torch

    from hpmc_b200 import datasets

    vols = datasets.batch_64()
    tensors = [torch.from_numpy(f).cuda() for f, _ in vols]
    b, offs, pos, nrm = _batch_run(hpmc, tensors, [iso for _, iso in vols], 1)
    for i in range(0, 64, 7):
        f, iso = vols[i]
        g = run_gpu(hpmc, f, iso, normals=1, capture_codes=False)
        assert offs[i + 1] - offs[i] == g["n"]
        np.testing.assert_allclose(pos[offs[i]:offs[i + 1]], g["pos"], rtol=0, atol=1e-6)
        np.testing.assert_allclose(nrm[offs[i]:offs[i + 1]], g["nrm"], rtol=0, atol=1e-6)
    b.close()


def test_autotune_choice_is_cached_per_signature(hpmc):
    """A second batch with the same volumes, scalar type and normal mode takes
    the first one's tuning without timing the candidates again."""
    import time

    import torch

    from hpmc_b200 import datasets

    vols = [datasets.metaballs(0, np.array([[0.5, 0.5, 0.5]]), np.array([0.2]), shape=(36 + 4 * i, 40, 44))
            for i in range(5)]
    fields = [torch.from_numpy(v).cuda() for v in vols]
    cap = 200000
    pos = torch.empty((cap, 4), dtype=torch.float32, device="cuda")
    nrm = torch.empty_like(pos)
    a = hpmc.Batch(fields, [1.0] * 5, normals=hpmc.NORMALS_CENTRAL)
    b = hpmc.Batch(fields, [1.0] * 5, normals=hpmc.NORMALS_CENTRAL)
    torch.cuda.synchronize()
    # only the two autotune calls are timed (creating a batch allocates)
    t0 = time.perf_counter()
    first = a.autotune(pos, nrm, cap)
    t1 = time.perf_counter()
    second = b.autotune(pos, nrm, cap)
    t2 = time.perf_counter()
    assert second == first == b.tuning()
    assert (t2 - t1) < 0.2 * (t1 - t0)
    b.extract(pos, nrm, cap)
    assert b.offsets()[-1] > 0
    a.close()
    b.close()
