"""Headless ports of the reference's apps (hpmc_b200/apps/*.cpp): C++ callers
that use HPMC's call sequences through the C ABI.  CPU: they build and reject
bad arguments before touching CUDA.  GPU: their vertex counts and .ply output
equal the oracle's / the handle path's on the same field and iso-value."""
from __future__ import annotations

import os
import struct
import subprocess

import numpy as np
import pytest

from hpmc_b200 import build as B


@pytest.fixture(scope="module")
def apps():
    return {name: B.app_path(name) for name in B.APPS if os.path.exists(B.app_path(name))}


def test_apps_built(apps):
    assert sorted(apps) == sorted(B.APPS), "run hpmc_b200.build.build_apps()"


@pytest.mark.parametrize("name,args", [("texture3d", ["64", "64"]), ("cayley", ["1", "2"]),
                                       ("metaballs", ["1", "2"]), ("transform_feedback", ["1", "2"]),
                                       ("custom_functor", ["1", "2"])])
def test_apps_reject_bad_arguments(apps, name, args):
    r = subprocess.run([apps[name], *args], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "Usage" in r.stderr


def _run(path, args):
    r = subprocess.run([path, *args, "--quiet"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return int(r.stdout.strip().split()[-1])


def _read_ply(path):
    with open(path, "rb") as f:
        head = b""
        while not head.endswith(b"end_header\n"):
            head += f.read(1)
        n = int([ln for ln in head.split(b"\n") if ln.startswith(b"element vertex")][0].split()[-1])
        v = np.frombuffer(f.read(24 * n), np.float32).reshape(n, 6)
    return v[:, :3], v[:, 3:]


@pytest.mark.gpu
def test_texture3d_app(apps, oracle, hpmc, tmp_path):
    from hpmc_b200 import datasets
    from tests.gpu_helpers import run_gpu

    vol, _ = datasets.noise_u8(48, seed=9)
    raw = tmp_path / "vol.raw"
    vol.tofile(raw)
    ply = tmp_path / "out.ply"
    n = _run(apps["texture3d"], ["48", "48", "48", str(raw), "--frames", "3", "--iso", "0.5", "--ply", str(ply)])
    g = run_gpu(hpmc, vol, 0.5, unorm=True, capture_codes=False)
    fz, fy, fx = vol.shape
    L = oracle.layout((fx, fy, fz))
    _, total = oracle.pyramid(oracle.codes(vol, L, 0.5, unorm=True), L)
    assert n == total == g["n"]
    p, q = _read_ply(ply)
    np.testing.assert_allclose(p, g["pos"][:, :3], rtol=0, atol=1e-6)
    np.testing.assert_allclose(q, g["nrm"][:, :3], rtol=0, atol=1e-6)


@pytest.mark.gpu
def test_cayley_app_binary_gradient(apps, oracle, hpmc, tmp_path):
    from tests.gpu_helpers import run_gpu

    ply = tmp_path / "c.ply"
    n = _run(apps["cayley"], ["40", "--frames", "2", "--iso", "0.25", "--ply", str(ply)])
    F = oracle.Functor("hpmc:cayley", [], (40, 40, 40))
    L = oracle.layout((40, 40, 40))
    _, total = oracle.pyramid(oracle.codes(F, L, 0.25, binary=True), L)
    assert n == total
    g = run_gpu(hpmc, F, 0.25, binary=True, gradient=True, capture_codes=False)
    p, q = _read_ply(ply)
    np.testing.assert_allclose(p, g["pos"][:, :3], rtol=0, atol=1e-6)
    np.testing.assert_allclose(q, g["nrm"][:, :3], rtol=0, atol=1e-6)


@pytest.mark.gpu
def test_metaballs_app_first_frame(apps, oracle, hpmc, tmp_path):
    """Frame 0 (t = 0): the app's uniforms are {0, centres at t = 0}."""
    from tests.gpu_helpers import run_gpu

    ply = tmp_path / "m.ply"
    n = _run(apps["metaballs"], ["48", "--frames", "1", "--ply", str(ply)])
    params = [0.0]
    for i in range(8):
        params += [np.float32(0.5 + 0.3 * np.sin(0.0)), np.float32(0.5 + 0.3 * np.cos(0.0)),
                   np.float32(0.5 + 0.3 * np.cos(0.0))]
    F = oracle.Functor("hpmc:twist_metaballs", [float(v) for v in params], (48, 48, 48))
    g = run_gpu(hpmc, F, 10.0, capture_codes=False)
    assert n == g["n"]
    p, _ = _read_ply(ply)
    np.testing.assert_allclose(p, g["pos"][:, :3], rtol=0, atol=1e-6)


@pytest.mark.gpu
def test_transform_feedback_app(apps, oracle, hpmc, tmp_path):
    from tests.gpu_helpers import compare, oracle_expect, run_gpu

    ply = tmp_path / "tf.ply"
    n = _run(apps["transform_feedback"], ["36", "--frames", "4", "--iso", "0.2", "--ply", str(ply)])
    F = oracle.Functor("hpmc:cayley", [], (36, 36, 36))
    g = run_gpu(hpmc, F, 0.2, gradient=True)
    e = oracle_expect(oracle, F, 0.2, normals=oracle.NORMALS_GRADIENT)
    compare(g, e)
    assert n == e["total"]
    p, q = _read_ply(ply)
    np.testing.assert_allclose(p, g["pos"][:, :3], rtol=0, atol=1e-6)
    np.testing.assert_allclose(q, g["nrm"][:, :3], rtol=0, atol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("flags,normals", [([], 0), (["--central"], 1), (["--gradient"], 2),
                                           (["--gradient", "--central"], 3)])
def test_custom_functor_app_matches_oracle(apps, oracle, tmp_path, flags, normals):
    """A caller's own functor type (hpmc_b200/apps/custom_functor.cu: a torus,
    compiled with include/hpmc_functor.cuh into the app's device code and
    registered as "app:torus") against the oracle's restatement of the same
    functor: the vertex count exactly, every vertex in order within the
    parity tolerances (positions 1e-5 of the spacing + 4 ulp, normals 1e-5 rad)."""
    from tests.gpu_helpers import angle, oracle_expect

    shape = (56, 40, 48)  # (z, y, x)
    ply = tmp_path / "torus.ply"
    n = _run(apps["custom_functor"], ["48", "40", "56", "--iso", "0", "--frames", "2", "--ply", str(ply), *flags])
    F = oracle.Functor("app:torus", [0.5, 0.25], shape)
    e = oracle_expect(oracle, F, 0.0, normals=normals)
    assert n == e["total"] > 0
    p, q = _read_ply(ply)
    spacing = 1.0 / np.array(e["L"].cells, np.float64)
    dp = np.abs(p.astype(np.float64) - e["pos"])
    assert (dp <= 1e-5 * spacing + 4 * np.finfo(np.float32).eps * np.abs(e["pos"])).all()
    ang, _, nb = angle(q, e["nrm"])
    ok = nb > 1e-6 * nb.max()
    assert ang[ok].max() <= 1e-5
