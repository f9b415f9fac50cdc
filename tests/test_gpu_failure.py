"""Failure detection without a GPU fault: the classifier's bounded waits.

The TMA column classifier waits on mbarriers for its field boxes; every wait
gives up after a time limit, the CTA drains the copies it has in flight and
the build reports a timeout.  These tests make a wait run out on purpose
through a test hook (HPMCsetTestStall / HPMCbatchSetTestStall): the producer
never issues one box -- neither its expected byte count nor its copy -- so
nothing is in flight for it, nothing faults, and the consumers' waits end by
their (lowered, 1 ms) limit.  The tests then check that the error reaches
the caller through the documented calls and that the handle and the CUDA
context stay usable: the next build, with the hook off, equals the oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from tests.gpu_helpers import compare, oracle_expect, run_gpu

pytestmark = pytest.mark.gpu

WAIT_US = 1000  # lowered wait limit: the timed-out build ends in a few milliseconds


def test_handle_build_timeout_is_reported_and_recoverable(hpmc, oracle):
    import torch

    from hpmc_b200 import _capi, datasets

    field_np, iso = datasets.cayley(96)
    dev = torch.device("cuda:0")
    field = torch.from_numpy(field_np).to(dev)
    stream = torch.cuda.Stream(device=dev)
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(stream)
    hp.set_field_device(field)
    hp.build(iso)
    n_ok = hp.acquire_number_of_vertices()
    assert hp.classify_path() == 1  # the TMA column classifier (the one with mbarrier waits)

    th = hpmc.TraversalHandle(hp)
    pos = torch.zeros((n_ok, 4), dtype=torch.float32, device=dev)
    nrm = torch.zeros_like(pos)
    th.set_buffers(pos, nrm, n_ok)

    # at 96^3 every persistent CTA streams one one-box column: each skips its box 0
    hp.set_test_stall(0, WAIT_US)
    hp.build(iso)
    assert hp.acquire_number_of_vertices() == 0
    assert hp.last_error == _capi.ERR_TIMEOUT
    # the handle is broken until it is reconfigured: the next calls refuse
    assert th.extract() is False
    assert hp.acquire_number_of_vertices() == 0

    # hook off, handle reconfigured (a field setter un-breaks it): correct again
    hp.set_test_stall(-1)
    hp.set_field_device(field)
    hp.build(iso)
    assert hp.acquire_number_of_vertices() == n_ok
    assert hp.last_error == 0
    assert hp.device_status() == 0
    th.close()
    hp.close()
    # and the context serves a full parity run
    g = run_gpu(hpmc, field_np, iso, normals=1)
    compare(g, oracle_expect(oracle, field_np, iso, normals=1))


def test_timeout_of_a_later_box_and_the_device_status(hpmc):
    import torch

    from hpmc_b200 import _capi, datasets

    field_np, iso = datasets.cayley(256)
    field = torch.from_numpy(field_np).cuda()
    hp = hpmc.HistoPyramid(hpmc.default_constants())
    hp.set_stream(torch.cuda.current_stream())
    hp.set_field_device(field)
    # at 256^3 2,368 one-box columns are shared by 296 persistent CTAs, so
    # some CTA streams at least 8 boxes: its box 5 comes after several refills
    # of the two ring slots
    hp.set_test_stall(5, WAIT_US)
    hp.build(iso)
    torch.cuda.synchronize()
    assert hp.device_status() & 8  # kStatusTimeout, read (and cleared) without acquiring
    hp.set_test_stall(-1)
    hp.set_field_device(field)
    hp.build(iso)
    assert hp.acquire_number_of_vertices() > 0
    assert hp.last_error == _capi.OK


def test_batch_timeout_is_reported_and_recoverable(hpmc):
    import torch

    from hpmc_b200 import _capi, datasets

    dev = torch.device("cuda:0")
    vols = [datasets.cayley(64), datasets.cayley(96)]
    fields = [torch.from_numpy(f).to(dev) for f, _ in vols]
    b = hpmc.Batch(fields, [iso for _, iso in vols], normals=hpmc.NORMALS_CENTRAL)
    b.set_tuning(63, 0, 0)  # 64-layer columns: 8 boxes per brick, box 2 is a ring refill
    cap = 400000
    pos = torch.zeros((cap, 4), dtype=torch.float32, device=dev)
    nrm = torch.zeros_like(pos)
    b.extract(pos, nrm, cap)
    ref = b.offsets()
    ref_pos = pos[: ref[-1]].clone()

    b.set_test_stall(1, 2, WAIT_US)
    b.extract(pos, nrm, cap)
    with pytest.raises(hpmc.HPMCError) as ei:
        b.offsets()
    assert ei.value.status == _capi.ERR_TIMEOUT

    b.set_test_stall(1, -1)
    pos.zero_()
    b.extract(pos, nrm, cap)
    assert b.offsets() == ref
    assert torch.equal(pos[: ref[-1]], ref_pos)
    with pytest.raises(hpmc.HPMCError):
        b.set_test_stall(7, 0)  # no such volume
    b.close()
