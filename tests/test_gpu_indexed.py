"""Indexed (welded) output, HPMCextractVerticesIndexed: one vertex per crossed
lattice edge in first-occurrence order of the soup, one index per soup
vertex.  Checked against the soup of the same build (HPMCextractVertices with
the per-vertex cell/edge debug output): the indices reproduce the soup
exactly and each unique vertex carries its soup vertices' values."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _soup_and_indexed(hpmc, field, iso, normals=0, binary=False, unorm=False):
    import torch

    f = torch.from_numpy(np.ascontiguousarray(field)).cuda()
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(torch.cuda.current_stream())
    hp.set_field_device(f, unorm=unorm)
    if binary:
        hp.set_field_as_binary()
    hp.set_normal_mode(normals)
    hp.build(iso)
    n = hp.acquire_number_of_vertices()
    th = hpmc.TraversalHandle(hp)
    m = max(n, 1)
    pos = torch.zeros((m, 4), device="cuda")
    nrm = torch.zeros_like(pos)
    info = torch.zeros((m, 4), dtype=torch.int32, device="cuda")
    th.set_debug_buffers(info, None)
    th.extract_to(pos, nrm, n)
    th.set_debug_buffers(None, None)
    upos = torch.full((m, 4), float("nan"), device="cuda")
    unrm = torch.full_like(upos, float("nan"))
    idx = torch.full((m,), 0xFFFFFFFF, dtype=torch.int64, device="cuda").to(torch.int32)
    nu, ni = th.extract_indexed(upos, unrm, idx, m, m)
    torch.cuda.synchronize()
    out = dict(n=n, nu=nu, ni=ni, pos=pos[:n].cpu().numpy(), nrm=nrm[:n].cpu().numpy(),
               info=info[:n].cpu().numpy(), upos=upos[:nu].cpu().numpy(), unrm=unrm[:nu].cpu().numpy(),
               idx=idx[:n].cpu().numpy().view(np.uint32))
    th.close()
    hp.close()
    return out


def _expected(oracle, shape, g):
    fz, fy, fx = shape
    et = oracle.edge_table()[(g["info"][:, 3] >> 16) & 0xff]
    a = g["info"][:, :3].astype(np.int64) + et[:, :3].astype(np.int64)
    key = ((a[:, 2] * fy + a[:, 1]) * fx + a[:, 0]) * 3 + et[:, 3].astype(np.int64)
    _, first, inv = np.unique(key, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    return rank[inv], first[order]


CASES = ["metaballs_64", "ties_u8", "cayley_f32", "binary"]


def _case(name):
    from hpmc_b200 import datasets

    if name == "metaballs_64":
        f, iso = datasets.metaballs_64()
        return f, iso, dict(normals=1)
    if name == "ties_u8":
        rng = np.random.default_rng(8)
        return rng.integers(100, 156, size=(30, 41, 52)).astype(np.uint8), 128.0, dict(normals=0)
    if name == "cayley_f32":
        f, iso = datasets.cayley(96)
        return f, iso, dict(normals=1)
    f, iso = datasets.metaballs_64()  # binary field: midpoints and table normals
    return f, iso, dict(binary=True)


@pytest.mark.parametrize("name", CASES)
def test_indexed_output_reproduces_soup(hpmc, oracle, name):
    field, iso, kw = _case(name)
    g = _soup_and_indexed(hpmc, field, iso, **kw)
    assert g["n"] > 0 and g["ni"] == g["n"]
    idx, first = _expected(oracle, field.shape, g)
    assert g["nu"] == len(first) < g["n"]  # welding removes duplicates
    np.testing.assert_array_equal(g["idx"], idx)
    np.testing.assert_allclose(g["upos"], g["pos"][first], rtol=0, atol=1e-6)
    np.testing.assert_allclose(g["unrm"], g["nrm"][first], rtol=0, atol=1e-6)
    # the indexed mesh is the soup
    np.testing.assert_allclose(g["upos"][g["idx"]], g["pos"], rtol=0, atol=1e-6)


def test_indexed_capacity(hpmc):
    import torch

    from hpmc_b200 import HPMCError, datasets

    f, iso = datasets.metaballs_64()
    t = torch.from_numpy(f).cuda()
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(torch.cuda.current_stream())
    hp.set_field_device(t)
    hp.build(iso)
    n = hp.acquire_number_of_vertices()
    th = hpmc.TraversalHandle(hp)
    small = torch.zeros((16, 4), device="cuda")
    idx = torch.zeros((n,), dtype=torch.int32, device="cuda")
    with pytest.raises(HPMCError):
        th.extract_indexed(small, None, idx)
    th.close()
    hp.close()
