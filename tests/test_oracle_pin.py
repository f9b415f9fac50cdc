"""The oracle, pinned to the reference's own code (CPU only).

* layout: the reference's HPMCdetermineLayout (hpmc/src/init.cpp:72-149),
  compiled from the HPMC sources into oracle/_ref/, against the oracle's
  restatement and the product's (HPMCgetLayout needs a GPU; the product's
  restatement is checked in the GPU tests);
* tables: the reference's tables.cpp arrays, and the derived HPMC-order
  tables checked for topological consistency;
* classification / pyramid / traversal: the oracle against brute-force numpy
  restatements and the committed golden fixtures.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


LAYOUT_CASES = [(32, 32, 32), (36, 36, 36), (64, 64, 64), (100, 100, 100), (128, 128, 128),
                (192, 192, 192), (256, 256, 256), (301, 301, 301), (512, 512, 512), (301, 324, 56),
                (3, 3, 3), (4, 4, 4), (5, 7, 9), (9, 9, 9), (16384, 3, 3), (3, 16384, 7), (1000, 20, 3)]


@pytest.mark.parametrize("lattice", LAYOUT_CASES)
def test_layout_matches_reference(oracle, lattice):
    mine = oracle.layout(lattice)
    ref = oracle.ref_layout(lattice)
    assert mine is not None and ref is not None
    assert mine.tile + mine.layout + (mine.size_l2, mine.size) == ref


def test_layout_random_matches_reference(oracle):
    rng = np.random.default_rng(7)
    for _ in range(3000):
        lat = [int(v) for v in rng.integers(3, 2000, 3)]
        cells = [int(rng.integers(2, v)) for v in lat]
        mine = oracle.layout(lat, cells)
        ref = oracle.ref_layout(lat, cells)
        assert (mine is None) == (ref is None)
        if mine:
            assert mine.tile + mine.layout + (mine.size_l2, mine.size) == ref


@pytest.mark.parametrize("lat,cells", [((1, 5, 5), None), ((16385, 4, 4), None), ((8, 8, 8), (8, 7, 7)),
                                       ((8, 8, 8), (7, 9, 7))])
def test_layout_rejections_match_reference(oracle, lat, cells):
    assert oracle.layout(lat, cells) is None
    assert oracle.ref_layout(lat, cells) is None


def test_one_cell_axis_is_defined(oracle):
    # The reference shifts by a negative amount for a 1-cell axis (undefined
    # behaviour, init.cpp:106-111); the restatement clamps the exponent at 0.
    L = oracle.layout((2, 2, 2))
    assert L.tile == (1, 1) and L.size == 1


def test_raw_tables_are_the_references(oracle):
    tri, edge, mid = oracle.ref_tables()
    assert tri.shape == (256, 16) and (tri[0] == -1).all() and (tri[255] == -1).all()
    # edge table: shift xyz in {0,1}, axis in {0,1,2}, and the shifted cube edge stays in the cube
    assert set(np.unique(edge[:, :3])) <= {0.0, 1.0} and set(np.unique(edge[:, 3])) <= {0.0, 1.0, 2.0}
    for e in range(12):
        a = edge[e, :3].copy()
        b = a.copy()
        b[int(edge[e, 3])] += 1
        assert b.max() <= 1.0
        assert np.allclose(mid[e], 0.5 * (a + b))


def test_derived_tables_topologically_consistent(oracle):
    """Every vertex of HPMC code c lies on an edge whose end points straddle the
    iso-surface under c's bit convention (bit dx+2dy+4dz) -- this pins
    remapCode (constants.cpp:42-50) and the edge decode (constants.cpp:255-264)."""
    count, eidx, ed, edn = oracle.tables()
    _, edge, _ = oracle.ref_tables()
    for c in range(256):
        assert (count[c] == 0) == (c in (0, 255))
        assert count[c] % 3 == 0
        for k in range(count[c]):
            e = eidx[c, k]
            a = edge[e, :3].astype(int)
            b = a.copy()
            b[int(edge[e, 3])] += 1
            bit_a = (c >> (a[0] + 2 * a[1] + 4 * a[2])) & 1
            bit_b = (c >> (b[0] + 2 * b[1] + 4 * b[2])) & 1
            assert bit_a != bit_b, (c, k, e)
            assert tuple(ed[c, k]) == tuple(edge[e])
    # every crossing edge of a case is used by some vertex
    for c in range(1, 255):
        crossing = set()
        for e in range(12):
            a = edge[e, :3].astype(int)
            b = a.copy()
            b[int(edge[e, 3])] += 1
            if ((c >> (a[0] + 2 * a[1] + 4 * a[2])) & 1) != ((c >> (b[0] + 2 * b[1] + 4 * b[2])) & 1):
                crossing.add(e)
        assert set(eidx[c, : count[c]].tolist()) == crossing


def test_product_table_generator_matches_oracle(oracle):
    import sys

    sys.path.insert(0, os.path.join(ROOT, "hpmc_b200", "csrc"))
    import gen_tables as G

    tri, edge, mid = oracle.ref_tables()
    cnt, ei, bn = G.derive(tri, edge, mid)
    oc, oei, _, oedn = oracle.tables()
    assert (cnt == oc).all() and (ei == oei).all()
    fr = oedn[:, :15, :3] - np.floor(oedn[:, :15, :3])
    assert np.array_equal((np.float32(2) * fr - np.float32(1)).astype(np.float32), bn[:, :15])


def test_every_mixed_case_has_vertices(oracle):
    """The classifier lists a cell as active iff its 8 corners are neither all
    inside nor all outside, without a table lookup.  That is exact only if the
    reference's count table gives every such case at least one triangle (a
    listed cell with no vertices would shift the traversal's cell mapping)."""
    cnt, _, _, _ = oracle.tables()
    cnt = np.asarray(cnt).reshape(256)
    assert cnt[0] == 0 and cnt[255] == 0
    assert (cnt[1:255] >= 3).all() and (cnt % 3 == 0).all() and cnt.max() <= 15


def _brute_codes(field, iso, cells):
    cx, cy, cz = cells
    f = field.astype(np.float64) if field.dtype != np.uint8 else field.astype(np.float32)
    below = (f < iso)
    code = np.zeros((cz, cy, cx), np.int32)
    for b in range(8):
        dx, dy, dz = b & 1, (b >> 1) & 1, (b >> 2) & 1
        code |= below[dz:dz + cz, dy:dy + cy, dx:dx + cx].astype(np.int32) << b
    return code.astype(np.uint8)


@pytest.mark.parametrize("shape", [(5, 7, 9), (9, 9, 9), (17, 33, 12), (40, 3, 21)])
def test_oracle_codes_brute_force(oracle, shape):
    rng = np.random.default_rng(sum(shape))
    fz, fy, fx = shape
    field = rng.integers(0, 4, size=shape).astype(np.float32)  # many ties at iso 2
    field[0, 0, 0] = np.nan
    L = oracle.layout((fx, fy, fz))
    codes = oracle.codes(field, L, 2.0)
    assert np.array_equal(codes, _brute_codes(field, 2.0, L.cells))


def test_oracle_pyramid_and_traversal_brute_force(oracle):
    rng = np.random.default_rng(11)
    for shape in [(6, 9, 7), (12, 5, 33), (20, 20, 20), (3, 3, 3)]:
        fz, fy, fx = shape
        field = rng.normal(size=shape).astype(np.float32)
        L = oracle.layout((fx, fy, fz))
        codes = oracle.codes(field, L, 0.0)
        levels, total = oracle.pyramid(codes, L)
        count, eidx, _, _ = oracle.tables()
        # brute force: cells sorted by Morton key, each emitting count[code] vertices
        cells = []
        for z in range(L.cells[2]):
            for y in range(L.cells[1]):
                for x in range(L.cells[0]):
                    cells.append((oracle.cell_key(L, x, y, z), x, y, z))
        cells.sort()
        expect = []
        for _, x, y, z in cells:
            c = codes[z, y, x]
            for k in range(count[c]):
                expect.append((x, y, z, c, k, eidx[c, k]))
        assert total == len(expect)
        cell, code, k, edge = oracle.traverse(codes, levels, L, 0, total)
        got = list(zip(cell[:, 0], cell[:, 1], cell[:, 2], code, k, edge))
        assert [tuple(int(v) for v in g) for g in got] == [tuple(int(v) for v in e) for e in expect]
        # every level is the 4-way sum of the one below
        for j in range(1, L.size_l2 + 2):
            assert np.array_equal(levels[j], levels[j - 1].reshape(-1, 4).sum(1, dtype=np.uint64).astype(np.uint32))


def test_level0_texture_encoding(oracle):
    rng = np.random.default_rng(3)
    field = rng.normal(size=(7, 10, 9)).astype(np.float32)
    L = oracle.layout((9, 10, 7))
    codes = oracle.codes(field, L, 0.1)
    tex = oracle.level0_texture(codes, L)
    count, _, _, _ = oracle.tables()
    levels, _ = oracle.pyramid(codes, L)
    # floor of the base texels = level-0 counts; channel c of texel (i,j) = key 4*morton(i,j)+c
    for j in range(L.size):
        for i in range(L.size):
            tu, tv = i // L.tile[0], j // L.tile[1]
            slice_ = tu + L.layout[0] * tv
            t = tex[j, i]
            if slice_ >= L.cells[2]:
                assert tuple(t) == (0.0, 0.0, np.float32(0.4), 0.0)
                continue
            for c in range(4):
                x = 2 * (i % L.tile[0]) + (c & 1)
                y = 2 * (j % L.tile[1]) + (c >> 1)
                if x < L.cells[0] and y < L.cells[1]:
                    code = codes[slice_, y, x]
                    assert np.floor(t[c]) == count[code]
                    assert int(round((t[c] - np.floor(t[c])) * 256 - 0.5)) == code
                    assert levels[0][oracle.cell_key(L, x, y, slice_)] == count[code]
                else:
                    assert t[c] == 0.0


def test_golden_fixtures(oracle):
    """Oracle output equals the committed fixtures (tests/golden/make_golden.py)."""
    files = sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz"))
    assert files, "no golden fixtures"
    from tests.golden import make_golden

    for fname in files:
        g = np.load(os.path.join(GOLDEN, fname))
        case = make_golden.CASES[fname[:-4]]
        out = make_golden.run_case(oracle, **case)
        for key in g.files:
            if g[key].dtype.kind == "f":
                np.testing.assert_allclose(out[key], g[key], rtol=0, atol=1e-12, err_msg=f"{fname}:{key}")
            else:
                assert np.array_equal(out[key], g[key]), f"{fname}:{key}"
