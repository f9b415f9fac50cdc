"""Functor fields (HPMCsetFieldCustom with a registered device functor, the
stand-in for the reference's custom GLSL fetch) against the oracle's FP32
restatement of the same functors.

The device functors round every operation like the oracle's plain FP32 C, so
case indices, pyramid levels, counts and the vertex order are bit-exact as for
array fields; geometry within the parity tolerances.  Gradient mode
(HPMCsetFieldCustom(..., GL_TRUE)) takes t from the functor values at the edge
ends and the normal from the analytic gradient: n = iso - lerp(grad) in the
default (forward) normal mode, as the reference computes it
(shadergen.cpp:539-551), and -lerp(grad) in central mode.
"""
from __future__ import annotations

import numpy as np
import pytest

from tests.gpu_helpers import compare, oracle_expect, run_gpu

pytestmark = pytest.mark.gpu


def _metaball_params(seed, n):
    rng = np.random.default_rng(seed)
    p = [float(n)]
    for _ in range(n):
        p += [float(v) for v in rng.uniform(0.2, 0.8, 3)] + [float(rng.uniform(0.05, 0.15))]
    return p


CASES = {
    "cayley_33": ("hpmc:cayley", [], (33, 33, 33), 0.1),
    "cayley_odd": ("hpmc:cayley", [], (20, 41, 37), -0.3),
    "cayley_64": ("hpmc:cayley", [], (64, 64, 64), 0.0),
    "metaballs_48": ("hpmc:metaballs", _metaball_params(1, 8), (48, 48, 48), 1.0),
    "metaballs_odd": ("hpmc:metaballs", _metaball_params(2, 5), (30, 50, 70), 1.2),
    "spheres_40": ("hpmc:spheres", _metaball_params(3, 6), (40, 40, 40), 0.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("normals", [0, 1])
def test_functor_fields_match_oracle(hpmc, oracle, name, normals):
    fname, params, shape, iso = CASES[name]
    F = oracle.Functor(fname, params, shape)
    g = run_gpu(hpmc, F, iso, normals=normals)
    e = oracle_expect(oracle, F, iso, normals=normals)
    assert g["path"] == 0  # functors take the generic classifier
    compare(g, e)


@pytest.mark.parametrize("shape,iso", [((33, 33, 33), 0.1), ((48, 40, 56), -0.2), ((64, 64, 64), 0.5)])
@pytest.mark.parametrize("normals", [0, 1])
def test_gradient_mode_matches_oracle(hpmc, oracle, shape, iso, normals):
    F = oracle.Functor("hpmc:cayley", [], shape)
    g = run_gpu(hpmc, F, iso, normals=normals, gradient=True)
    e = oracle_expect(oracle, F, iso, normals=oracle.NORMALS_GRADIENT + normals)
    compare(g, e)


def test_gradient_mode_binary_field(hpmc, oracle):
    """apps/cayley's configuration: gradient snippet, binary field (table normals)."""
    F = oracle.Functor("hpmc:cayley", [], (48, 48, 48))
    g = run_gpu(hpmc, F, 0.3, binary=True, gradient=True)
    e = oracle_expect(oracle, F, 0.3, binary=True)
    compare(g, e, binary=True)


def test_twisted_metaballs_close_to_oracle(hpmc, oracle):
    """sin/cos round differently on the device and the host: the counts agree
    to within the cells whose samples lie within a few ulps of iso."""
    params = [2.5] + [v for i in range(8) for v in (0.5 + 0.3 * np.sin(i), 0.5 + 0.3 * np.cos(0.9 * i),
                                                    0.5 + 0.3 * np.cos(0.7 * i))]
    F = oracle.Functor("hpmc:twist_metaballs", params, (48, 48, 48))
    g = run_gpu(hpmc, F, 10.0)
    e = oracle_expect(oracle, F, 10.0)
    assert e["total"] > 1000
    assert abs(g["n"] - e["total"]) <= 0.01 * e["total"]
    assert np.count_nonzero(g["codes"] != e["codes"]) <= 0.001 * g["codes"].size


@pytest.mark.parametrize("shape", [(21, 34, 30), (40, 48, 64)])
@pytest.mark.parametrize("normals", [0, 1, 2, 3])
def test_rgba_gradient_textures_match_oracle(hpmc, oracle, shape, normals):
    """HPMCsetFieldTexture3D on an RGBA float texture (HPMC_SCALAR_F32X4:
    gradient in .xyz, the field in .w).  Modes 0/1: forward/central
    differences of the value channel; 2/3: the stored gradient
    (shadergen.cpp:260-266, 539-551), n = iso - lerp(grad) or -lerp(grad)."""
    rng = np.random.default_rng(sum(shape) + normals)
    field = rng.normal(size=shape + (4,)).astype(np.float32)
    field[..., 3][rng.random(shape) < 0.05] = 0.5  # ties with iso
    iso = 0.5
    gradient = normals >= 2
    g = run_gpu(hpmc, field, iso, normals=normals % 2, gradient=gradient, texture=True)
    e = oracle_expect(oracle, field, iso, normals=normals)
    assert g["path"] == 0  # float4 fields take the generic classifier
    compare(g, e)


def test_gradient_mode_on_a_scalar_texture_reads_zero_gradient(hpmc, oracle):
    """A single-channel texture in gradient mode: GL's alpha texture reads
    rgb = 0, so the reference's normal is iso - 0 = iso (scaled); the oracle
    restates that."""
    rng = np.random.default_rng(8)
    field = rng.normal(size=(20, 22, 24)).astype(np.float32)
    g = run_gpu(hpmc, field, 0.25, gradient=True, texture=True)
    e = oracle_expect(oracle, field, 0.25, normals=oracle.NORMALS_GRADIENT)
    compare(g, e)
