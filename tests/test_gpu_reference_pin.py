"""The GPU against the reference's own arithmetic at the benchmark workload.

The reference's generated GLSL passes (oracle/glsl_pin.py: the shader text
its generator emits, compiled for the CPU) run on the 512 x 512 x 33 z-slab
of the 512^3 FP32 Cayley benchmark field, and the product extracts the same
slab on the GPU with the reference's forward-difference normals.  Required:
the same vertex count; the same cells, edges and crossing parameters in the
same order (the reference's positions equal the shader's own tile arithmetic
applied to the GPU's cell, edge and t per vertex, to the FP32 rounding of that
arithmetic --
tests/reference_positions.py explains the reference's 6-digit texel constant);
normals within 1e-5 relative; and the GPU's positions within the parity
tolerance of the lattice-exact ones (1e-5 of the spacing plus 4 ulp).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_benchmark_slab_matches_reference_glsl(hpmc, oracle):
    import torch

    from hpmc_b200 import datasets
    from oracle import glsl_pin
    from tests.reference_positions import printed_texel_constant, reference_positions, shader_rounding

    slab, iso = datasets.cayley(512, slices=33)  # bit-identical to the benchmark field's first 33 slices
    fz, fy, fx = slab.shape
    _, n_ref, pos_ref, nrm_ref = glsl_pin.run(slab, iso, max_vertices=1 << 21, keep_levels=False)

    dev = torch.device("cuda:0")
    f = torch.from_numpy(slab).to(dev)
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(torch.cuda.current_stream())
    hp.set_field_device(f)
    hp.set_normal_mode(hpmc.NORMALS_FORWARD)
    hp.build(iso)
    n = hp.acquire_number_of_vertices()
    assert n == n_ref > 0
    th = hpmc.TraversalHandle(hp)
    pos = torch.empty((n, 4), dtype=torch.float32, device=dev)
    nrm = torch.empty_like(pos)
    info = torch.empty((n, 4), dtype=torch.int32, device=dev)
    tt = torch.empty((n,), dtype=torch.float32, device=dev)
    th.set_debug_buffers(info, tt)
    assert th.extract_to(pos, nrm, n) == n
    torch.cuda.synchronize()
    pos, nrm, info, tt = pos.cpu().numpy(), nrm.cpu().numpy(), info.cpu().numpy(), tt.cpu().numpy()
    th.close()
    hp.close()

    L = oracle.layout((fx, fy, fz))
    cell = info[:, :3]
    edge = (info[:, 3] >> 16) & 0xff
    c_printed = printed_texel_constant(oracle.ref_glsl(5, (fx, fy, fz)))
    model = reference_positions(L, cell, edge, tt.astype(np.float64), oracle.edge_table(), c_printed)
    spacing = 1.0 / np.array(L.cells, np.float64)
    # same cells, edges and t, in the same order: the reference's positions are its tile
    # arithmetic on the GPU's (cell, edge, t), to FP32 rounding of that arithmetic
    assert (np.abs(pos_ref - model) <= 4e-6 * (np.abs(model) + spacing) + shader_rounding(L)).all()
    # forward-difference normals of the same samples
    scale = np.abs(nrm_ref).max(1, keepdims=True) + 1e-30
    assert (np.abs(nrm[:, :3] - nrm_ref) <= 1e-5 * scale).all()
    # and the GPU's own positions are lattice-exact: a[axis] + t on the edge
    e = oracle.edge_table()[edge]
    exact = (cell + e[:, :3]).astype(np.float64)
    exact[np.arange(n), e[:, 3].astype(int)] += tt
    exact *= spacing
    assert (np.abs(pos[:, :3] - exact) <= 1e-5 * spacing + 4 * np.finfo(np.float32).eps * np.abs(exact)).all()
