"""CUDA path vs the oracle through the C ABI (needs a B200).

Topology (case indices, every dense pyramid level, the vertex count and the
vertex -> (cell, k, edge) order) must be bit-exact.  Geometry: the edge
parameter t within 1e-5 (cell-local), positions within 1e-5 of the lattice
spacing plus 4 FP32 ulps of the world coordinate, normals within 1e-5 rad of
the FP64 oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from tests.golden import make_golden
from tests.gpu_helpers import compare, oracle_expect, run_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(make_golden.CASES))
@pytest.mark.parametrize("normals", [0, 1])
def test_golden_cases(hpmc, oracle, name, normals):
    case = make_golden.CASES[name]
    field = make_golden.make_field(case["kind"], case["shape"], case["seed"])
    kw = dict(cells=case.get("cells"), extent=case.get("extent", (1.0, 1.0, 1.0)),
              binary=case.get("binary", False), unorm=case.get("unorm", False))
    g = run_gpu(hpmc, field, case["iso"], normals=normals, **kw)
    e = oracle_expect(oracle, field, case["iso"], normals=normals, **kw)
    compare(g, e, extent=kw["extent"], binary=kw["binary"])
    # the committed fixtures agree with both
    gold = np.load(__import__("os").path.join(make_golden.HERE, name + ".npz"))
    assert int(gold["total"][0]) == g["n"]
    assert np.array_equal(gold["cell"], g["info"][:, :3])


SHAPES = [(3, 3, 3), (4, 5, 6), (9, 9, 9), (5, 7, 9), (40, 3, 21), (17, 33, 12), (33, 33, 33), (34, 65, 66),
          (70, 40, 100), (64, 64, 64), (48, 128, 36)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("dtype", ["f32", "u8"])
def test_random_lattices(hpmc, oracle, shape, dtype):
    rng = np.random.default_rng(sum(shape) * 7 + (0 if dtype == "f32" else 1000))
    if dtype == "f32":
        field = rng.normal(size=shape).astype(np.float32)
        field[rng.random(shape) < 0.05] = 0.0  # exact ties with iso 0
        iso = 0.0
    else:
        field = rng.integers(100, 156, size=shape).astype(np.uint8)
        iso = 128.0
    g = run_gpu(hpmc, field, iso)
    e = oracle_expect(oracle, field, iso)
    compare(g, e)


TMA_SHAPES = [(2, 50, 36), (7, 65, 68), (33, 31, 40), (100, 33, 64), (40, 40, 48), (2, 64, 64), (9, 100, 96),
              (70, 200, 144)]


@pytest.mark.parametrize("shape", TMA_SHAPES)
@pytest.mark.parametrize("dtype", ["f32", "u8", "unorm8"])
def test_tma_column_path(hpmc, oracle, shape, dtype):
    """Aligned fields whose 32x32 blocks lie inside one slice tile take the TMA
    column kernel (odd cell counts, single-slice volumes, partial footprints)."""
    rng = np.random.default_rng(sum(shape) * 3 + len(dtype))
    if dtype == "f32":
        field = rng.normal(size=shape).astype(np.float32)
        field[rng.random(shape) < 0.05] = 0.0
        iso = 0.0
    else:
        field = rng.integers(100, 156, size=shape).astype(np.uint8)
        iso = 128.0 if dtype == "u8" else 128.0 / 255.0
    unorm = dtype == "unorm8"
    g = run_gpu(hpmc, field, iso, unorm=unorm)
    L = oracle.layout((shape[2], shape[1], shape[0]))
    expect_tma = 2 * L.tile[0] >= 32 and 2 * L.tile[1] >= 32 and (shape[2] * field.itemsize) % 16 == 0
    assert g["path"] == (1 if expect_tma else 0)
    e = oracle_expect(oracle, field, iso, unorm=unorm)
    compare(g, e)


@pytest.mark.parametrize("pad", [1, 3, 16])
def test_pitched_fields_take_generic_path_identically(hpmc, oracle, pad):
    rng = np.random.default_rng(pad)
    field = rng.normal(size=(40, 36, 70)).astype(np.float32)
    g = run_gpu(hpmc, field, 0.1, pitch_pad=pad)
    e = oracle_expect(oracle, field, 0.1)
    compare(g, e)


def test_grid_smaller_than_lattice(hpmc, oracle):
    rng = np.random.default_rng(5)
    field = rng.normal(size=(30, 50, 70)).astype(np.float32)
    cells = (50, 40, 20)
    g = run_gpu(hpmc, field, 0.0, cells=cells, extent=(1.0, 2.0, 3.0))
    e = oracle_expect(oracle, field, 0.0, cells=cells, extent=(1.0, 2.0, 3.0))
    compare(g, e, extent=(1.0, 2.0, 3.0))


def test_config_metaballs_64(hpmc, oracle):
    from hpmc_b200 import datasets

    field, iso = datasets.metaballs_64()
    for normals in (0, 1):
        g = run_gpu(hpmc, field, iso, normals=normals)
        e = oracle_expect(oracle, field, iso, normals=normals)
        rep = compare(g, e)
        assert rep["n"] > 50000


def test_config_spheres_128(hpmc, oracle):
    from hpmc_b200 import datasets

    field, iso = datasets.spheres_sdf()
    g = run_gpu(hpmc, field, iso, normals=1)
    e = oracle_expect(oracle, field, iso, normals=1)
    compare(g, e)


@pytest.mark.slow
def test_config_noise_u8_256_ties(hpmc, oracle):
    """uint8 256^3 with ~256k samples equal to the iso-value: >2^24 vertices."""
    from hpmc_b200 import datasets

    field, iso = datasets.noise_u8()
    assert int((field == 128).sum()) > 100000
    g = run_gpu(hpmc, field, iso, normals=1)
    e = oracle_expect(oracle, field, iso, normals=1)
    rep = compare(g, e)
    assert rep["n"] > 2**24


@pytest.mark.slow
def test_config_cayley_512_full_size(hpmc, oracle):
    """The benchmark workload at its full size (FP32 512^3 Cayley cubic, iso 0,
    central normals, the TMA column path): every case index, every dense
    level, the count, the vertex order and the geometry of all vertices; a
    second build + extraction is bit-identical (the persistent traversal's
    dynamic work assignment does not change the output)."""
    from hpmc_b200 import datasets

    field, iso = datasets.cayley(512)
    g = run_gpu(hpmc, field, iso, normals=1)
    assert g["path"] == 1  # the TMA column classifier
    e = oracle_expect(oracle, field, iso, normals=1)
    rep = compare(g, e)
    assert rep["n"] > 3_000_000
    g2 = run_gpu(hpmc, field, iso, normals=1, capture_codes=False)
    assert g2["n"] == g["n"]
    assert np.array_equal(g2["pos"].view(np.uint32), g["pos"].view(np.uint32))
    assert np.array_equal(g2["nrm"].view(np.uint32), g["nrm"].view(np.uint32))


def test_product_layout_matches_oracle(hpmc, oracle):
    """The product's own HPMCdetermineLayout (init.cpp:72-149) against the
    oracle's, which is pinned to the reference's compiled init.cpp: the
    survey's sizes, 300 random lattices and grids, and the sizes the
    reference rejects (an axis below 2 or above 16384 samples, a grid not
    smaller than the lattice), which fail lazily with HPMC_ERR_LAYOUT."""
    import torch

    from hpmc_b200 import _capi

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(23)
    cases = [((32, 32, 32), None), ((36, 36, 36), None), ((64, 64, 64), None), ((128, 128, 128), None),
             ((192, 192, 192), None), ((301, 301, 301), None), ((301, 324, 56), None), ((2, 2, 2), None),
             ((16384, 2, 2), None), ((2, 16384, 2), None), ((2, 2, 16384), None), ((3, 3, 3), None),
             ((16385, 2, 2), None), ((2, 2, 16385), None), ((1, 5, 5), None), ((8, 8, 8), (8, 7, 7)),
             ((8, 8, 8), (7, 9, 7))]
    while len(cases) < 317:
        lat = tuple(int(v) for v in np.exp(rng.uniform(np.log(2), np.log(400), 3)).astype(int) + 1)
        if lat[0] * lat[1] * lat[2] > 4_000_000:
            continue
        cells = None if rng.random() < 0.5 else tuple(int(rng.integers(1, v)) for v in lat)
        cases.append((lat, cells))
    c = hpmc.default_constants()
    rejected = 0
    for lat, cells in cases:
        t = torch.zeros((lat[2], lat[1], lat[0]), dtype=torch.float32, device=dev)
        hp = hpmc.HistoPyramid(c)
        hp.set_field_device(t)
        if cells is not None:
            hp.set_grid_size(*cells)
        exp = oracle.layout(lat, cells)
        try:
            got = tuple(hp.layout())
        except hpmc.HPMCError:
            got = None
            assert hp.last_error == _capi.ERR_LAYOUT, (lat, cells)
        if exp is None:
            rejected += 1
            assert got is None, (lat, cells, got)
        else:
            assert got == exp.tile + exp.layout + (exp.size_l2, exp.size), (lat, cells, got)
        hp.close()
    assert rejected >= 5


def test_caller_kernels_on_the_stream_stay_ordered(hpmc, oracle):
    """The build and extraction launch with programmatic stream serialization.
    A caller's kernel that rewrites the field right before a build, or the
    output right after an extraction, on the same stream must still be fully
    ordered with them: alternate two fields through one device buffer."""
    import torch

    from hpmc_b200 import datasets

    dev = torch.device("cuda:0")
    fa, iso = datasets.cayley(96)
    fb = np.ascontiguousarray(fa[:, :, ::-1] * np.float32(1.5) + np.float32(0.01))
    ea = oracle_expect(oracle, fa, iso, normals=1)
    eb = oracle_expect(oracle, fb, iso, normals=1)
    assert ea["total"] != eb["total"]
    src = [torch.from_numpy(fa).to(dev), torch.from_numpy(fb).to(dev)]
    exp = [ea, eb]
    buf = torch.empty_like(src[0])
    stream = torch.cuda.Stream(device=dev)
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(stream)
    hp.set_field_device(buf)
    hp.set_normal_mode(1)
    th = hpmc.TraversalHandle(hp)
    cap = max(ea["total"], eb["total"])
    pos = torch.empty((cap, 4), dtype=torch.float32, device=dev)
    nrm = torch.empty((cap, 4), dtype=torch.float32, device=dev)
    th.set_buffers(pos, nrm, cap)
    for i in range(6):
        e = exp[i % 2]
        with torch.cuda.stream(stream):
            torch.mul(src[i % 2], 1.0, out=buf)  # a kernel, not a copy
        hp.build(iso)
        n = hp.acquire_number_of_vertices()
        assert n == e["total"], (i, n, e["total"])
        th.extract()
        with torch.cuda.stream(stream):
            snap = pos[:n].clone()  # a kernel reading the output right after the extraction
            pos.fill_(float("nan"))
        stream.synchronize()
        dp = np.abs(snap[:, :3].cpu().numpy().astype(np.float64) - e["pos"])
        assert dp.max() <= 1e-5 / 95 + 1e-6, (i, dp.max())
    th.close()
    hp.close()


def test_retaint_between_extractions_stays_stream_ordered(hpmc, oracle):
    """A setter that taints the handle (here the grid extent) between an
    asynchronous extraction and the next build must not disturb the
    extraction still in flight: the lazy set-up clears the pyramid and the
    control block in stream order.  No host sync between the two volumes,
    on a non-blocking stream."""
    import torch

    from hpmc_b200 import datasets

    dev = torch.device("cuda:0")
    fa, iso = datasets.cayley(256)
    fb = np.ascontiguousarray(fa[::-1, :, :] * np.float32(1.25) - np.float32(0.02))
    ext_b = (2.0, 1.5, 0.75)
    ea = oracle_expect(oracle, fa, iso, normals=1)
    eb = oracle_expect(oracle, fb, iso, normals=1, extent=ext_b)
    ta, tb = torch.from_numpy(fa).to(dev), torch.from_numpy(fb).to(dev)
    stream = torch.cuda.Stream(device=dev)
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(stream)
    hp.set_normal_mode(1)
    hp.set_field_device(ta)
    th = hpmc.TraversalHandle(hp)
    pa = torch.full((ea["total"], 4), float("nan"), dtype=torch.float32, device=dev)
    na = torch.full_like(pa, float("nan"))
    pb = torch.full((eb["total"], 4), float("nan"), dtype=torch.float32, device=dev)
    nb = torch.full_like(pb, float("nan"))
    torch.cuda.synchronize()
    for _ in range(3):
        hp.set_field_device(ta)
        hp.set_grid_extent(1.0, 1.0, 1.0)  # taints: set-up runs at the next build
        hp.build(iso)
        th.extract_to(pa, na, ea["total"], sync=False)
        hp.set_grid_extent(*ext_b)  # taints again while A's extraction is in flight
        hp.set_field_device(tb)
        hp.build(iso)
        th.extract_to(pb, nb, eb["total"], sync=False)
    stream.synchronize()
    for pos, e, ext in ((pa, ea, (1.0, 1.0, 1.0)), (pb, eb, ext_b)):
        spacing = np.array(ext) / np.array(e["L"].cells, np.float64)
        dp = np.abs(pos[:, :3].cpu().numpy().astype(np.float64) - e["pos"])
        assert (dp <= 1e-5 * spacing[None, :] + 4 * np.finfo(np.float32).eps * np.abs(e["pos"])).all()
    th.close()
    hp.close()


def test_builds_overlapping_extractions_use_alternate_sets(hpmc, oracle):
    """A build on the column path may start while the previous extraction of
    the same pyramid still runs (the traversal lets it launch early): builds
    alternate between two sets of levels and arena, so the running
    extraction keeps reading its own.  Two different fields back to back,
    no host sync and no set-up in between, on a non-blocking stream."""
    import torch

    from hpmc_b200 import datasets

    dev = torch.device("cuda:0")
    fa, iso = datasets.cayley(256)
    fb = np.ascontiguousarray(fa[:, ::-1, :] * np.float32(0.8) + np.float32(0.03))
    ea = oracle_expect(oracle, fa, iso, normals=1)
    eb = oracle_expect(oracle, fb, iso, normals=1)
    assert ea["total"] != eb["total"]
    ta, tb = torch.from_numpy(fa).to(dev), torch.from_numpy(fb).to(dev)
    stream = torch.cuda.Stream(device=dev)
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(stream)
    hp.set_normal_mode(1)
    hp.set_field_device(ta)
    th = hpmc.TraversalHandle(hp)
    outs = [[torch.full((e["total"], 4), float("nan"), dtype=torch.float32, device=dev) for _ in range(2)]
            for e in (ea, eb) for _ in range(3)]
    torch.cuda.synchronize()
    for i in range(3):
        for j, (t, e) in enumerate(((ta, ea), (tb, eb))):
            hp.set_field_device(t)
            hp.build(iso)
            assert hp.classify_path() == 1
            p, n = outs[3 * j + i]
            th.extract_to(p, n, e["total"], sync=False)
    stream.synchronize()
    for j, e in enumerate((ea, eb)):
        for i in range(3):
            got = outs[3 * j + i][0][:, :3].cpu().numpy().astype(np.float64)
            dp = np.abs(got - e["pos"])
            assert np.isfinite(got).all() and dp.max() <= 1e-5 / 255 + 1e-6, (j, i, dp.max())
    th.close()
    hp.close()


def test_build_on_previous_extraction_output_waits_for_it(hpmc, oracle):
    """A field that is the previous extraction's output buffer: the build must
    not start before that extraction ends (its field bytes overlap the
    extraction's outputs, so it takes the ordinary ordered path).  The second
    volume, of the same lattice (no set-up in between), is the first one's
    position buffer read as a 256^3 FP32 field (2.0, above the iso-value 0.5,
    past the vertices)."""
    import torch

    from hpmc_b200 import datasets

    dev = torch.device("cuda:0")
    fa, iso = datasets.cayley(256)
    ta = torch.from_numpy(fa).to(dev)
    cap = 256 ** 3 // 4  # the position buffer holds exactly one 256^3 FP32 field
    stream = torch.cuda.Stream(device=dev)
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(stream)
    hp.set_normal_mode(1)
    hp.set_field_device(ta)
    th = hpmc.TraversalHandle(hp)
    pa = torch.full((cap, 4), 2.0, dtype=torch.float32, device=dev)
    na = torch.empty_like(pa)
    field_b = pa.view(256, 256, 256)
    # the second volume's field and expected output, from an ordered first pass
    hp.build(iso)
    na_ = th.extract_to(pa, na, cap)
    assert 0 < na_ < cap
    fb = field_b.cpu().numpy()
    eb = oracle_expect(oracle, fb, 0.5, normals=1)
    pb = torch.empty((eb["total"], 4), dtype=torch.float32, device=dev)
    nb = torch.empty_like(pb)
    for _ in range(2):
        with torch.cuda.stream(stream):
            pa.fill_(2.0)
        hp.set_field_device(ta)
        hp.build(iso)
        th.extract_to(pa, na, cap, sync=False)
        hp.set_field_device(field_b)  # the extraction above is still writing it
        hp.build(0.5)
        assert hp.classify_path() == 1
        nv = th.extract_to(pb, nb, eb["total"])
        assert nv == eb["total"], (nv, eb["total"])
        dp = np.abs(pb[:, :3].cpu().numpy().astype(np.float64) - eb["pos"])
        assert dp.max() <= 1e-5 / 255 + 1e-6, dp.max()
    th.close()
    hp.close()


def test_binary_mode_and_feedback_capture(hpmc, oracle):
    """Binary fields (midpoints + table normals) and the N3F_V3F capture."""
    import torch

    rng = np.random.default_rng(9)
    field = rng.random((20, 22, 24)).astype(np.float32)
    g = run_gpu(hpmc, field, 0.0, binary=True)
    e = oracle_expect(oracle, field, 0.0, binary=True)
    compare(g, e, binary=True)
    # transform-feedback layout through the reference entry point
    dev = torch.device("cuda:0")
    t = torch.from_numpy(field).to(dev)
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(torch.cuda.current_stream())
    hp.set_field_device(t)
    hp.set_field_as_binary()
    hp.build(0.0)
    n = hp.acquire_number_of_vertices()
    th = hpmc.TraversalHandle(hp)
    fb = torch.zeros(n * 6, dtype=torch.float32, device=dev)
    th.set_feedback_buffer(fb, n)
    assert th.extract_feedback()
    torch.cuda.synchronize()
    fb = fb.cpu().numpy().reshape(n, 6)
    np.testing.assert_array_equal(fb[:, 3:], g["pos"][:, :3])
    np.testing.assert_array_equal(fb[:, :3], g["nrm"][:, :3])


def test_reference_call_sequence_and_errors(hpmc):
    """The reference's API sequence (texture3d app, apps/texture3d/texture3d.cpp:144-221)
    with a registered device field standing in for the GL texture."""
    import ctypes as C

    import torch

    from hpmc_b200 import _capi

    L = hpmc.lib()
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(1)
    vol = torch.from_numpy(rng.integers(0, 255, size=(24, 20, 16)).astype(np.uint8)).to(dev)
    c = L.HPMCcreateConstants(4, 3)
    assert c
    h = L.HPMCcreateHistoPyramid(c)
    assert L.HPMCacquireNumberOfVertices(h) == 0  # broken until configured (hpiface.cpp:57)
    name = L.HPMCregisterDeviceField(vol.data_ptr(), _capi.SCALAR_UNORM8, 16, 20, 24, 0, 0)
    L.HPMCsetLatticeSize(h, 16, 20, 24)
    L.HPMCsetGridSize(h, 15, 19, 23)
    L.HPMCsetGridExtent(h, 16 / 24, 20 / 24, 1.0)
    L.HPMCsetFieldTexture3D(h, name, 0)
    th = L.HPMCcreateTraversalHandle(h)
    assert th
    assert L.HPMCgetTraversalShaderFunctions(th) is None
    assert L.HPMCgetLastError(h) == _capi.ERR_UNSUPPORTED
    assert L.HPMCsetTraversalHandleProgram(th, 1, 0, 1, 2) is False
    assert L.HPMCextractVertices(th) is False  # no output buffers bound
    L.HPMCbuildHistopyramid(h, 0.5)
    n = L.HPMCacquireNumberOfVertices(h)
    assert n > 0
    pos = torch.empty((n, 4), dtype=torch.float32, device=dev)
    nrm = torch.empty((n, 4), dtype=torch.float32, device=dev)
    assert L.HPMCsetTraversalHandleBuffers(th, pos.data_ptr(), nrm.data_ptr(), n) == 0
    assert L.HPMCextractVertices(th) is True
    # too-small buffers: first `capacity` vertices written, HPMC_ERR_CAPACITY reported
    small = torch.full((5, 4), -7.0, dtype=torch.float32, device=dev)
    assert L.HPMCsetTraversalHandleBuffers(th, small.data_ptr(), None, 5) == 0
    assert L.HPMCextractVertices(th) is False
    assert L.HPMCgetLastError(h) == _capi.ERR_CAPACITY
    torch.cuda.synchronize()
    np.testing.assert_array_equal(small.cpu().numpy(), pos[:5].cpu().numpy())
    st = C.c_uint(0)
    assert L.HPMCgetDeviceStatus(h, C.byref(st)) == 0 and (st.value & 2)
    # a bad layout fails lazily like the reference (init.cpp:98-103)
    L.HPMCsetGridSize(h, 16, 19, 23)
    assert L.HPMCcreateTraversalHandle(h) is None
    assert L.HPMCgetLastError(h) == _capi.ERR_LAYOUT
    L.HPMCdestroyTraversalHandle(th)
    L.HPMCdestroyHandle(h)
    L.HPMCunregisterDeviceField(name)
    L.HPMCdestroyConstants(c)


def test_custom_fetch_name_rules(hpmc):
    from hpmc_b200 import _capi

    L = hpmc.lib()
    c = L.HPMCcreateConstants(4, 3)
    h = L.HPMCcreateHistoPyramid(c)
    L.HPMCsetLatticeSize(h, 16, 16, 16)
    L.HPMCsetFieldCustom(h, b"float HPMC_fetch(vec3 p) { return p.x; }", 0, 0)
    assert L.HPMCgetLastError(h) == _capi.ERR_UNSUPPORTED
    assert L.HPMCgetBuilderProgram(h) == 0  # broken
    L.HPMCsetFieldCustom(h, b"hpmc:cayley", 0, 0)
    assert L.HPMCgetBuilderProgram(h) != 0
    L.HPMCdestroyHandle(h)
    L.HPMCdestroyConstants(c)
