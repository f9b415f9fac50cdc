"""Adjoint of the extraction on the GPU (HPMCextractVerticesAdjoint and the
torch.autograd.Function over it) against the oracle's FP64 adjoint and FP64
central finite differences.

Workload: the 128^3 signed-distance field of 16 spheres, iso 0, loss
L = sum_v w_v . p_v + u_v . n_v with w, u ~ N(0, 1) per vertex.

Tolerances: against the FP64 adjoint, |g - g64| <= 1e-5 * S + 1e-9 * max|g64|
per sample, S = the sum of |terms| that reach the sample (FP32 rounding and
atomic reordering of those terms).  Against finite differences with
h = 1e-4 on 1000 samples whose +-h perturbation keeps every case fixed:
|g - fd(h)| <= 4 |fd(h) - fd(h/2)| + 1e-4 |fd| + 1e-5 * S (the first term
bounds the O(h^2) truncation error of the central difference).
"""
from __future__ import annotations

import numpy as np
import pytest

from tests.adjoint_helpers import choose_samples, fd_gradients

pytestmark = pytest.mark.gpu


def _setup(oracle, field, iso):
    O = oracle
    fz, fy, fx = field.shape
    L = O.layout((fx, fy, fz))
    codes = O.codes(field, L, iso)
    levels, total = O.pyramid(codes, L)
    cell, code, k, edge = O.traverse(codes, levels, L, 0, total)
    return L, total, cell, code, k, edge


def _gpu_grad(hpmc, field_np, iso, normals, w, u, extent=(1.0, 1.0, 1.0)):
    import torch

    from hpmc_b200 import autograd

    f = torch.from_numpy(field_np).cuda().requires_grad_(True)
    pos, nrm = autograd.extract(f, iso, normals=normals, extent=extent)
    wt = torch.from_numpy(w).cuda()
    ut = torch.from_numpy(u).cuda()
    loss = (pos * wt).sum() + (nrm * ut).sum()
    loss.backward()
    torch.cuda.synchronize()
    return pos.shape[0], f.grad.double().cpu().numpy()


@pytest.fixture(scope="module")
def spheres():
    from hpmc_b200 import datasets

    return datasets.spheres_sdf(128)


@pytest.mark.parametrize("normals", [0, 1])
def test_adjoint_matches_fp64_adjoint(hpmc, oracle, spheres, normals):
    field, iso = spheres
    L, total, cell, code, k, edge = _setup(oracle, field, iso)
    rng = np.random.default_rng(42 + normals)
    # float4 cotangents; the w components are random and must be ignored
    w = rng.normal(size=(total, 4)).astype(np.float32)
    u = rng.normal(size=(total, 4)).astype(np.float32)
    n, g = _gpu_grad(hpmc, field, iso, normals, w, u)
    assert n == total
    g64, S = oracle.adjoint(field.astype(np.float64), L, iso, cell, edge, w[:, :3], u[:, :3],
                            normal_mode=normals, with_abs=True)
    err = np.abs(g - g64)
    tol = 1e-5 * S + 1e-9 * np.abs(g64).max()
    assert (err <= tol).all(), float((err / np.maximum(tol, 1e-30)).max())
    assert np.count_nonzero(g) > 0.5 * np.count_nonzero(g64)


@pytest.mark.parametrize("normals", [1, 0])
def test_adjoint_finite_differences(hpmc, oracle, spheres, normals):
    field, iso = spheres
    L, total, cell, code, k, edge = _setup(oracle, field, iso)
    rng = np.random.default_rng(7 + normals)
    w = rng.normal(size=(total, 4)).astype(np.float32)
    u = rng.normal(size=(total, 4)).astype(np.float32)
    _, g = _gpu_grad(hpmc, field, iso, normals, w, u)
    _, S = oracle.adjoint(field.astype(np.float64), L, iso, cell, edge, w[:, :3], u[:, :3], normal_mode=normals,
                          with_abs=True)
    h = 1e-4
    samples = choose_samples(oracle, field, iso, cell, edge, 1000, 123, h, central=normals == 1)
    assert len(samples) == 1000
    dp = w[:, :3].astype(np.float64)
    dn = u[:, :3].astype(np.float64)
    fd1 = fd_gradients(oracle, field, L, iso, cell, code, k, edge, dp, dn, normals, (1.0, 1.0, 1.0), samples, h)
    fd2 = fd_gradients(oracle, field, L, iso, cell, code, k, edge, dp, dn, normals, (1.0, 1.0, 1.0), samples,
                       h / 2)
    idx = np.array([s for s, _ in samples])
    gs = g.reshape(-1)[idx]
    tol = 4 * np.abs(fd1 - fd2) + 1e-4 * np.abs(fd1) + 1e-5 * S.reshape(-1)[idx] + 1e-12
    err = np.abs(gs - fd1)
    assert (err <= tol).all(), float((err / tol).max())
    # Richardson extrapolation: agreement well inside the truncation bound for most samples
    rich = (4 * fd2 - fd1) / 3
    rel = np.abs(gs - rich) / (np.abs(rich) + 1e-3 * np.abs(rich).max())
    assert np.median(rel) < 1e-4


def test_adjoint_accumulates_and_ignores_absent_cotangents(hpmc, oracle, spheres):
    import torch

    field, iso = spheres
    f = torch.from_numpy(field).cuda()
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(torch.cuda.current_stream())
    hp.set_field_device(f)
    hp.set_normal_mode(1)
    hp.build(iso)
    n = hp.acquire_number_of_vertices()
    th = hpmc.TraversalHandle(hp)
    pos = torch.empty((n, 4), device="cuda")
    nrm = torch.empty((n, 4), device="cuda")
    th.extract_to(pos, nrm, n)
    rng = np.random.default_rng(3)
    w = torch.from_numpy(rng.normal(size=(n, 4)).astype(np.float32)).cuda()
    d1 = torch.zeros_like(f)
    th.adjoint(w, None, n, d1)
    d2 = torch.zeros_like(f)
    th.adjoint(w, None, n, d2)
    th.adjoint(w, None, n, d2)
    torch.cuda.synchronize()
    np.testing.assert_allclose(d2.cpu().numpy(), 2 * d1.cpu().numpy(), rtol=1e-5, atol=1e-6 * float(d1.abs().max()))
    # positions only: the FP64 adjoint with zero normal cotangents
    L, total, cell, code, k, edge = _setup(oracle, field, iso)
    g64, S = oracle.adjoint(field.astype(np.float64), L, iso, cell, edge, w.cpu().numpy()[:, :3],
                            np.zeros((n, 3)), normal_mode=1, with_abs=True)
    err = np.abs(d1.double().cpu().numpy() - g64)
    assert (err <= 1e-5 * S + 1e-9 * np.abs(g64).max()).all()
    th.close()
    hp.close()


def test_adjoint_uint8_field(hpmc, oracle):
    import torch

    from hpmc_b200 import datasets

    field, iso = datasets.noise_u8(48, seed=5)
    L, total, cell, code, k, edge = _setup(oracle, field, iso)
    f = torch.from_numpy(field).cuda()
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(torch.cuda.current_stream())
    hp.set_field_device(f)
    hp.set_normal_mode(0)
    hp.build(iso)
    n = hp.acquire_number_of_vertices()
    assert n == total
    th = hpmc.TraversalHandle(hp)
    pos = torch.empty((n, 4), device="cuda")
    nrm = torch.empty((n, 4), device="cuda")
    th.extract_to(pos, nrm, n)
    rng = np.random.default_rng(8)
    w = rng.normal(size=(n, 4)).astype(np.float32)
    u = rng.normal(size=(n, 4)).astype(np.float32)
    d = torch.zeros(field.shape, dtype=torch.float32, device="cuda")
    th.adjoint(torch.from_numpy(w).cuda(), torch.from_numpy(u).cuda(), n, d)
    torch.cuda.synchronize()
    g64, S = oracle.adjoint(field, L, iso, cell, edge, w[:, :3], u[:, :3], normal_mode=0, with_abs=True)
    err = np.abs(d.double().cpu().numpy() - g64)
    assert (err <= 1e-5 * S + 1e-9 * np.abs(g64).max()).all()
    th.close()
    hp.close()


def test_autograd_handle_pool(hpmc, spheres):
    """The autograd wrapper reuses pyramid handles per field shape: two
    differentiable forwards of different fields in flight before either
    backward each keep their own pyramid (their gradients equal those computed
    one at a time, up to the atomics' summation order), and a forward without
    gradients hands its handles back at once."""
    import torch

    from hpmc_b200 import autograd

    field, iso = spheres
    base = torch.from_numpy(field).cuda()
    fields = [base, base * 1.1 + 0.002]

    def loss_of(pos, nrm, seed):
        g = torch.Generator(device="cpu").manual_seed(seed)
        w = torch.randn(pos.shape, generator=g).cuda()
        u = torch.randn(nrm.shape, generator=g).cuda()
        return (pos * w).sum() + (nrm * u).sum()

    alone = []
    for i, f in enumerate(fields):
        x = f.clone().requires_grad_(True)
        pos, nrm = autograd.extract(x, iso)
        loss_of(pos, nrm, i).backward()
        alone.append(x.grad.clone())
    xs = [f.clone().requires_grad_(True) for f in fields]
    outs = [autograd.extract(x, iso) for x in xs]  # both forwards before either backward
    for i in (1, 0):
        loss_of(*outs[i], i).backward()
    for x, g in zip(xs, alone):
        torch.testing.assert_close(x.grad, g, rtol=1e-5, atol=1e-6 * float(g.abs().max()))
    key = (str(base.device), tuple(base.shape), base.dtype, tuple(base.stride()))
    free = len(autograd._POOL[key])
    with torch.no_grad():
        autograd.extract(base, iso)
    assert len(autograd._POOL[key]) == free  # borrowed and given back
