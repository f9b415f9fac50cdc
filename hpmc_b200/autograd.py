"""Differentiable extraction: torch.autograd.Function over the C ABI.

forward  = HPMCbuildHistopyramid + HPMCextractVerticesToBuffers (float4
           positions and normals in the reference's vertex order);
backward = HPMCextractVerticesAdjoint, the hand-written adjoint kernel: it
           recomputes each vertex's traversal (nothing is stored between the
           passes besides the pyramid) and scatters dL/dp and dL/dn onto the
           field samples the vertex read, through
           t = (f_a - iso)/(f_a - f_b) and the normal stencil.

Topology is piecewise constant: the case indices and the vertex list do not
depend on the field's values between iso crossings, so the gradient is the
derivative of the geometry with the topology held fixed.  Only float32 array
fields are differentiable; the w components of the incoming gradients are
ignored (positions carry w = 1, normals w = 0).
"""
from __future__ import annotations

import torch

from . import (NORMALS_FORWARD, HistoPyramid, TraversalHandle, default_constants)


# Pyramid + traversal handles reused across calls, per (device, field shape,
# dtype, strides): a forward borrows a pair and gives it back right away when
# no gradient will be asked for, otherwise after its backward.  No device
# allocation per call once the pool holds a pair for the shape.
_POOL: dict = {}


def _borrow(field):
    key = (str(field.device), tuple(field.shape), field.dtype, tuple(field.stride()))
    free = _POOL.setdefault(key, [])
    if free:
        return key, free.pop()
    hp = HistoPyramid(default_constants())
    hp.set_field_device(field)  # sizes the pyramid once for this shape
    return key, (hp, TraversalHandle(hp))


def _give_back(key, handles):
    handles[0]._keep.clear()  # the pool does not keep the caller's field alive
    _POOL.setdefault(key, []).append(handles)


class ExtractFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, field, iso, normals, extent):
        key, (hp, th) = _borrow(field)
        hp.set_stream(torch.cuda.current_stream())
        hp.set_field_device(field)
        hp.set_grid_extent(*extent)
        hp.set_normal_mode(normals)
        hp.build(float(iso))
        n = hp.acquire_number_of_vertices()
        if hp.last_error:
            from . import HPMCError

            err = hp.last_error
            _give_back(key, (hp, th))
            raise HPMCError(err, "HPMCbuildHistopyramid")
        pos = torch.empty((n, 4), dtype=torch.float32, device=field.device)
        nrm = torch.empty((n, 4), dtype=torch.float32, device=field.device)
        if n:
            th.extract_to(pos, nrm, n, sync=False)
        ctx.n = n
        if ctx.needs_input_grad[0]:
            ctx.save_for_backward(field)
            ctx.handles = (key, hp, th)  # the pyramid of this forward, kept for the adjoint
        else:
            ctx.handles = None
            _give_back(key, (hp, th))
        return pos, nrm

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, gpos, gnrm):
        (field,) = ctx.saved_tensors
        key, hp, th = ctx.handles
        dfield = torch.empty_strided(field.shape, field.stride(), dtype=torch.float32, device=field.device)
        dfield.zero_()
        if ctx.n:
            gp = None if gpos is None else gpos.to(torch.float32).contiguous()
            gn = None if gnrm is None else gnrm.to(torch.float32).contiguous()
            hp.set_stream(torch.cuda.current_stream())
            th.adjoint(gp, gn, ctx.n, dfield)
        ctx.handles = None
        _give_back(key, (hp, th))
        return dfield, None, None, None


def extract(field: torch.Tensor, iso: float, *, normals: int = NORMALS_FORWARD, extent=(1.0, 1.0, 1.0)):
    """Differentiable extraction of a (z, y, x) float32 CUDA field: returns
    (positions, normals), each (n, 4) float32; gradients flow to `field`."""
    return ExtractFunction.apply(field, float(iso), int(normals), tuple(float(e) for e in extent))
