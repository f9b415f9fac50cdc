"""The oracle's FP64 adjoint (the reference gradient for the CUDA adjoint)
against FP64 central finite differences, on the CPU.

Perturbations keep every case fixed (the sample stays on its side of iso),
so the topology -- and the vertex list -- is constant and the loss is a
smooth function of the perturbed sample."""
from __future__ import annotations

import numpy as np
import pytest

from tests.adjoint_helpers import choose_samples, fd_gradients


def _spheres(n, seed):
    from hpmc_b200 import datasets

    f, iso = datasets.spheres_sdf(n, seed=seed, count=6)
    return f, iso


@pytest.mark.parametrize("normal_mode", [0, 1])
@pytest.mark.parametrize("extent", [(1.0, 1.0, 1.0), (2.0, 1.0, 0.5)])
def test_oracle_adjoint_matches_finite_differences(oracle, normal_mode, extent):
    O = oracle
    field, iso = _spheres(40, 11)
    fz, fy, fx = field.shape
    L = O.layout((fx, fy, fz))
    codes = O.codes(field, L, iso)
    levels, total = O.pyramid(codes, L)
    cell, code, k, edge = O.traverse(codes, levels, L, 0, total)
    assert total > 100
    rng = np.random.default_rng(5)
    dpos = rng.normal(size=(total, 3))
    dnrm = rng.normal(size=(total, 3))
    g = O.adjoint(field.astype(np.float64), L, iso, cell, edge, dpos, dnrm, normal_mode=normal_mode, extent=extent)
    h = 1e-6
    samples = choose_samples(O, field, iso, cell, edge, 300, 9, h, central=normal_mode == 1)
    fd = fd_gradients(O, field, L, iso, cell, code, k, edge, dpos, dnrm, normal_mode, extent, samples, h)
    gs = g.reshape(-1)[[s for s, _ in samples]]
    err = np.abs(gs - fd)
    assert (err <= 1e-6 * (np.abs(fd) + 1.0)).all(), float((err / (np.abs(fd) + 1.0)).max())


def test_oracle_adjoint_is_linear_in_the_cotangents(oracle):
    O = oracle
    field, iso = _spheres(24, 3)
    fz, fy, fx = field.shape
    L = O.layout((fx, fy, fz))
    codes = O.codes(field, L, iso)
    levels, total = O.pyramid(codes, L)
    cell, code, k, edge = O.traverse(codes, levels, L, 0, total)
    rng = np.random.default_rng(1)
    a1, a2 = rng.normal(size=(total, 3)), rng.normal(size=(total, 3))
    b1, b2 = rng.normal(size=(total, 3)), rng.normal(size=(total, 3))
    f64 = field.astype(np.float64)
    g1 = O.adjoint(f64, L, iso, cell, edge, a1, b1, normal_mode=1)
    g2 = O.adjoint(f64, L, iso, cell, edge, a2, b2, normal_mode=1)
    g12 = O.adjoint(f64, L, iso, cell, edge, a1 + 2 * a2, b1 + 2 * b2, normal_mode=1)
    np.testing.assert_allclose(g12, g1 + 2 * g2, rtol=1e-10, atol=1e-10 * np.abs(g12).max())
