"""Benchmark of the HistoPyramid marching-cubes hot path on B200.

Workload (one "step" = one extraction of one volume): FP32 512^3 Cayley cubic
16xyz + 4(x^2+y^2+z^2) - 1 + N(0, 1e-3) on [-1,1]^3, iso 0, central-difference
normals: classify + reduce (HPMCbuildHistopyramid) and traversal into float4
position/normal streams (HPMCextractVertices, vertex count read on the device).

  value    Gcells/s with the field resident in HBM (device time, CUDA events)
  e2e      the same through the public API with host buffers: pinned H2D of
           the field, build, count (host sync), extraction, D2H of every vertex;
           two volumes in flight (two handles on two streams: the H2D of
           volume k+1 overlaps volume k); the one-at-a-time figure beside it
  roofline the whole extraction step (classify + reduce + traverse) against
           the measured HBM copy bandwidth; algorithmic bytes = field bytes
           read once + 32 B per vertex written; the build and the traversal
           alone are reported beside it ("kernels")
  cpu_baseline  the reference's generated shader passes run as C++ on the host
           cores (the oracle restatement if they cannot be built), full volume
  batched  64 uneven FP32 volumes: batched extractor (CUDA-graph replay) vs
           the plain per-volume loop through the handle API (sync-free: device
           vertex counts, preallocated outputs; and the loop that reads every
           count on the host), volumes/s
  adjoint  128^3 sphere SDF: adjoint (backward) time over forward time

--impl reference times the reference's path on the host cores instead: the
reference is GLSL for a GL driver (no GL stack on this box), so the shader
text its generator emits is compiled for the CPU (oracle/glsl_pin.py, OpenMP
over all host threads) and run on the full 512^3 workload.  Its only normal
estimate is the forward difference; the repository arm reports a
forward-normal step beside its central-normal headline for that comparison.

N > 1 (torchrun): every rank extracts its own volume (independent objects,
no collective on the data path): weak scaling, value = all ranks' cells / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcells/s @512³ f32 (% HBM roof); batched vs plain vols/s; adjoint/fwd time"
WORKLOAD = ("cayley_512: FP32 512^3 lattice, Cayley cubic 16xyz+4(x^2+y^2+z^2)-1 + N(0,1e-3) on [-1,1]^3, "
            "iso 0, central-difference normals, float4 position+normal streams")
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes (read + write) of one build (classify_columns + reduce_levels)
# per field byte, and of one traversal per vertex, from ncu captures on the
# 384^3 Cayley field (226,492,416 field bytes, 2,092,962 vertices;
# profiles/classify_columns_cayley384.txt, profiles/reduce_levels_cayley384.txt,
# profiles/traverse_kernel_cayley384.txt).  Build traffic grows with the field
# and traversal traffic with the vertices, so the 512^3 figure is these
# ratios times the field bytes and the vertex count.
BUILD_TRAFFIC_PER_FIELD_BYTE = (226531840 + 6623488 + 1064704) / 226492416
TRAVERSE_TRAFFIC_PER_VERTEX = (29616896 + 15378688) / 2092962


NOMINAL_HBM_GBS = 8000.0  # B200 HBM3e nominal (DGX figure), reported beside the measured copy peak


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.path = None

    def start(self):
        import tempfile

        try:
            fd, self.path = tempfile.mkstemp(prefix="hpmc_clocks_", suffix=".csv")
            self.fh = os.fdopen(fd, "w")
            visible = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            gpu = visible.split(",")[self.gpu] if visible else str(self.gpu)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.fh, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.5)  # let nvidia-smi start sampling before the GPU work
        except Exception:
            self.proc = None
        return self

    def stop(self):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()
            with open(self.path) as f:
                self.lines = [ln.strip() for ln in f if ln.strip()]
            os.unlink(self.path)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _reference_volume(field_np, iso, threads, max_vertices):
    """One run of the reference's own passes -- the GLSL its shader generator
    emits, compiled for the CPU (oracle/glsl_pin.py) -- on the whole volume:
    base level, reductions, count and extractVertex for every vertex (forward
    normals, the reference's only estimate).  Returns (cells, vertices, threads)."""
    import os as _os

    from oracle import glsl_pin

    th = threads if threads > 0 else (_os.cpu_count() or 1)
    _, n, _, _ = glsl_pin.run(field_np, iso, max_vertices=max_vertices, keep_levels=False, threads=th)
    fz, fy, fx = field_np.shape
    return (fx - 1) * (fy - 1) * (fz - 1), n, th


def cpu_baseline(field_np, iso, max_vertices, threads=0, min_seconds=10.0):
    """The reference's path on the host cores: its generated shaders run as C++
    (kind "reference"); the oracle restatement (kind "port") if they cannot be
    built.  The whole workload, repeated for >= min_seconds."""
    from oracle import oracle as O

    try:
        _reference_volume(field_np, iso, threads, max_vertices)  # compile + warm
        kind = "reference"
    except Exception:
        kind = "port"
    fz, fy, fx = field_np.shape
    cells = (fx - 1) * (fy - 1) * (fz - 1)
    t0 = time.perf_counter()
    runs = 0
    verts = 0
    cores = threads if threads > 0 else O.max_threads()
    while True:
        if kind == "reference":
            _, verts, cores = _reference_volume(field_np, iso, threads, max_vertices)
        else:
            verts, _, _ = O.extract_count(field_np, iso, normal_mode=O.NORMALS_FORWARD, threads=threads,
                                          geometry=True)
        runs += 1
        if time.perf_counter() - t0 >= min_seconds:
            break
    dt = time.perf_counter() - t0
    what = ("the reference's generated GLSL passes compiled for the CPU (base level, reductions, count, "
            "extractVertex with forward normals)" if kind == "reference"
            else "oracle restatement (codes+pyramid+traversal+FP64 geometry, forward normals)")
    return {"value": cells * runs / dt / 1e9, "unit": "Gcells/s", "cores": cores, "kind": kind,
            "sample": f"the whole {fx}x{fy}x{fz} workload ({cells} cells, {verts} vertices), {what}, {runs} runs"}


def run_reference(args, rank, world):
    """The reference's path on the host cores (rank 0 only): its generated
    shaders compiled for the CPU, all host threads, the whole 512^3 workload
    per step."""
    if rank != 0:
        return
    from hpmc_b200 import datasets

    field, iso = datasets.cayley(args.lattice)
    max_vertices = 1 << 23 if args.lattice <= 512 else 1 << 26
    try:
        for _ in range(args.warmup):
            cells, verts, threads = _reference_volume(field, iso, 0, max_vertices)
        kind = "reference"
        step = lambda: _reference_volume(field, iso, 0, max_vertices)  # noqa: E731
    except Exception:
        from oracle import oracle as O

        kind = "port"
        threads = O.max_threads()
        fz, fy, fx = field.shape

        def step():
            n, _, _ = O.extract_count(field, iso, normal_mode=O.NORMALS_FORWARD, threads=threads, geometry=True)
            return (fx - 1) * (fy - 1) * (fz - 1), n, threads
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s0 = time.perf_counter()
        cells, verts, threads = step()
        vals.append(cells / (time.perf_counter() - s0) / 1e9)
    dt = time.perf_counter() - t0
    value = statistics.median(vals)
    sample = (f"the whole {args.lattice}^3 workload per step ({cells} cells, {verts} vertices): "
              + ("the reference's generated GLSL passes compiled for the CPU (forward normals)" if kind == "reference"
                 else "oracle restatement (forward normals)"))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Gcells/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": WORKLOAD, "lattice": [args.lattice] * 3},
            "cpu_baseline": {"value": value, "unit": "Gcells/s", "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "Gcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference runs its passes as GLSL in a GL driver, unavailable on this box (no GL stack); "
                    "its generated shader text is compiled and run on the host cores instead. Its only normal "
                    "estimate is the forward difference (the repository arm's forward_normals_step_ms is the "
                    "like-for-like figure)"}
    print(json.dumps(line), flush=True)


def run_batched(args, dev, stream, rank=0, world=1):
    """64 uneven FP32 metaball volumes: one CUDA-graph replay of the batched
    extractor vs the plain per-volume loop through the handle API, both on the
    same stream, CUDA events.  Two plain loops: the sync-free one (build, then
    HPMCextractVerticesToBuffers reading the vertex count on the device, into
    outputs allocated beforehand) and the one that reads every count on the
    host (build, acquire count, extract).  With N ranks each takes its share
    of the 64 volumes (greedy split by cells) and the time is the maximum
    over the ranks."""
    import torch
    import torch.distributed as dist

    import hpmc_b200 as H
    from hpmc_b200 import datasets, multi

    all_vols = datasets.batch_64()
    share = multi.split_volumes([f.size for f, _ in all_vols], world)[rank]
    vols = [all_vols[i] for i in share]
    tensors = [torch.from_numpy(f).to(dev) for f, _ in vols]
    isos = [iso for _, iso in vols]
    cells = sum((f.shape[0] - 1) * (f.shape[1] - 1) * (f.shape[2] - 1) for f, _ in vols)
    field_bytes = sum(f.nbytes for f, _ in vols)
    C = H.default_constants()
    # plain loop: one handle per volume, created and sized outside the timed region
    hps, ths, outs = [], [], []
    with torch.cuda.stream(stream):
        for t, iso in zip(tensors, isos):
            hp = H.HistoPyramid(C)
            hp.set_stream(stream)
            hp.set_field_device(t)
            hp.set_normal_mode(H.NORMALS_CENTRAL)
            hp.build(iso)
            n = hp.acquire_number_of_vertices()
            th = H.TraversalHandle(hp)
            pos = torch.empty((max(n, 1), 4), dtype=torch.float32, device=dev)
            nrm = torch.empty_like(pos)
            th.set_buffers(pos, nrm, n)
            hps.append(hp)
            ths.append(th)
            outs.append(n)
    total = sum(outs)

    def plain_sync():
        for hp, th, iso in zip(hps, ths, isos):
            hp.build(iso)
            hp.acquire_number_of_vertices()
            th.extract()

    def plain():  # sync-free: device counts, outputs sized beforehand
        for hp, th, iso, (p, q), n in zip(hps, ths, isos, bufs, outs):
            hp.build(iso)
            th.extract_to(p, q, n, sync=False)

    bufs = [th._keep["buf"] for th in ths]
    steps = max(3, min(args.steps, 20))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    loop_ms = {}
    for name, fn in (("sync_free", plain), ("host_sync", plain_sync)):
        with torch.cuda.stream(stream):
            for _ in range(3):
                fn()
            stream.synchronize()
            if world > 1:
                dist.barrier()
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
            stream.synchronize()
        loop_ms[name] = multi.max_over_ranks(e0.elapsed_time(e1) / steps, device=dev)
    plain_ms = loop_ms["sync_free"]

    b = H.Batch(tensors, isos, normals=H.NORMALS_CENTRAL)
    pos = torch.empty((total, 4), dtype=torch.float32, device=dev)
    nrm = torch.empty_like(pos)
    with torch.cuda.stream(stream):
        if args.batch_tuning:
            b.set_tuning(*[int(v) for v in args.batch_tuning.split(",")])
            tuning = b.tuning()
        else:
            tuning = b.autotune(pos, nrm, total, stream=stream)
        for _ in range(3):
            b.extract(pos, nrm, total, stream=stream)
        stream.synchronize()
        if world > 1:
            dist.barrier()
        e0.record(stream)
        for _ in range(steps):
            b.extract(pos, nrm, total, stream=stream)
        e1.record(stream)
        stream.synchronize()
    batched_ms = multi.max_over_ranks(e0.elapsed_time(e1) / steps, device=dev)
    offs = b.offsets()
    assert offs[-1] == total, (offs[-1], total)
    for th in ths:
        th.close()
    for hp in hps:
        hp.close()
    b.close()
    nall = len(all_vols)
    cells_all = sum((f.shape[0] - 1) * (f.shape[1] - 1) * (f.shape[2] - 1) for f, _ in all_vols)
    return {"workload": "batch_64: 64 FP32 volumes, edges log-uniform [32,192] (x4), 4-32 metaballs, iso U[0.8,1.5], "
                        "central normals",
            "volumes": nall, "cells": cells_all, "field_bytes": sum(f.nbytes for f, _ in all_vols),
            "vertices": int(multi.sum_over_ranks(total, device=dev)), "ranks": world,
            "plain_ms": plain_ms, "plain_host_sync_ms": loop_ms["host_sync"], "batched_ms": batched_ms,
            "plain_vols_per_s": nall / (plain_ms * 1e-3), "batched_vols_per_s": nall / (batched_ms * 1e-3),
            "speedup": plain_ms / batched_ms, "speedup_vs_host_sync_loop": loop_ms["host_sync"] / batched_ms,
            "plain_loop": "sync-free: per volume HPMCbuildHistopyramid + HPMCextractVerticesToBuffers "
                          "(device vertex count, outputs allocated beforehand)",
            "batched_gcells_per_s": cells_all / (batched_ms * 1e-3) / 1e9,
            "batched_hbm_fraction": (sum(f.nbytes for f, _ in all_vols) + 32 * total) / (batched_ms * 1e-3) / 1e9
            / hbm_peak()[0],
            "tuning": {"column_slices": tuning[0], "traverse_ctas_per_sm": tuning[1], "rounds": tuning[2]},
            "graph": True, "steps": steps}


def run_adjoint(args, dev, stream):
    """Differentiable extraction on the 128^3 SDF of 16 spheres (iso 0, central
    normals): forward = build + extraction, backward = zeroing dL/df + the
    adjoint kernel for L = sum w.p + u.n (w, u ~ N(0,1)); CUDA events.  The
    8 MB field stays in L2 for both passes."""
    import torch

    import hpmc_b200 as H
    from hpmc_b200 import datasets

    field_np, iso = datasets.spheres_sdf(128)
    f = torch.from_numpy(field_np).to(dev)
    hp = H.HistoPyramid(H.default_constants())
    hp.set_stream(stream)
    hp.set_field_device(f)
    hp.set_normal_mode(H.NORMALS_CENTRAL)
    hp.build(iso)
    n = hp.acquire_number_of_vertices()
    th = H.TraversalHandle(hp)
    pos = torch.empty((n, 4), dtype=torch.float32, device=dev)
    nrm = torch.empty_like(pos)
    th.set_buffers(pos, nrm, n)
    g = torch.Generator(device="cpu").manual_seed(4)
    w = torch.randn((n, 4), generator=g).to(dev)
    u = torch.randn((n, 4), generator=g).to(dev)
    dfield = torch.zeros_like(f)
    steps = max(5, min(args.steps, 50))

    def fwd():
        hp.build(iso)
        th.extract()

    def bwd():
        dfield.zero_()
        th.adjoint(w, u, n, dfield)

    res = {}
    with torch.cuda.stream(stream):
        for name, fn in (("forward", fwd), ("backward", bwd)):
            for _ in range(3):
                fn()
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
            stream.synchronize()
            res[name] = e0.elapsed_time(e1) / steps
    th.close()
    hp.close()
    return {"workload": "spheres_128: FP32 128^3 SDF of 16 spheres, iso 0, central normals, "
                        "L = sum w.p + u.n, w,u ~ N(0,1)",
            "vertices": n, "forward_ms": res["forward"], "backward_ms": res["backward"],
            "backward_over_forward": res["backward"] / res["forward"], "steps": steps,
            "l2": "8 MB field resident in L2 for both passes"}


def run_hpmc(args, rank, world, local_rank):
    import torch

    import hpmc_b200 as H
    from hpmc_b200 import datasets, multi

    dev = torch.device(f"cuda:{local_rank}")
    torch.cuda.set_device(dev)
    field_np, iso = datasets.cayley(args.lattice)
    fz, fy, fx = field_np.shape
    cells = (fx - 1) * (fy - 1) * (fz - 1)
    field_bytes = field_np.nbytes
    field = torch.from_numpy(field_np).to(dev)
    stream = torch.cuda.Stream(device=dev)

    C = H.Constants()
    hp = H.HistoPyramid(C)
    hp.set_stream(stream)
    hp.set_field_device(field)
    hp.set_normal_mode(H.NORMALS_CENTRAL)
    hp.build(iso)
    nverts = hp.acquire_number_of_vertices()
    th = H.TraversalHandle(hp)
    pos = torch.empty((nverts, 4), dtype=torch.float32, device=dev)
    nrm = torch.empty((nverts, 4), dtype=torch.float32, device=dev)
    th.set_buffers(pos, nrm, nverts)

    path = hp.classify_path()

    def step():
        hp.build(iso)
        th.extract()

    # clocks are sampled from the start of the warm-up to the end of the timed
    # region (a short timed region alone would fall between two samples)
    clocks = ClockSampler(local_rank).start()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    stream.synchronize()

    # --- timed region: field resident in HBM -------------------------------
    # K steps back to back with events only at the ends: an event recorded
    # between two launches costs several microseconds and cuts the launches'
    # programmatic overlap (~12 us per step measured at 512^3).
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t_begin = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_begin.record(stream)
    for _ in range(args.steps):
        step()
    t_end.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    total_ms = t_begin.elapsed_time(t_end)

    # --- kernel breakdown: a second pass of K steps with events around the
    # build (classify + reduce) and the extraction of every step
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3 * args.steps)]
    torch.cuda.synchronize()
    for i in range(args.steps):
        ev[3 * i].record(stream)
        hp.build(iso)
        ev[3 * i + 1].record(stream)
        th.extract()
        ev[3 * i + 2].record(stream)
    stream.synchronize()
    clocks.stop()
    build_ms = [ev[3 * i].elapsed_time(ev[3 * i + 1]) for i in range(args.steps)]
    trav_ms = [ev[3 * i + 1].elapsed_time(ev[3 * i + 2]) for i in range(args.steps)]
    # --- the same step with forward normals (the reference's only estimate),
    # timed like the headline loop, for the like-for-like comparison with the
    # reference arm
    hp.set_normal_mode(H.NORMALS_FORWARD)
    with torch.cuda.stream(stream):
        for _ in range(3):
            step()
    torch.cuda.synchronize()
    f_begin = torch.cuda.Event(enable_timing=True)
    f_end = torch.cuda.Event(enable_timing=True)
    f_begin.record(stream)
    for _ in range(args.steps):
        step()
    f_end.record(stream)
    stream.synchronize()
    fwd_ms = multi.max_over_ranks(f_begin.elapsed_time(f_end) / args.steps, device=dev)
    hp.set_normal_mode(H.NORMALS_CENTRAL)

    total_ms = multi.max_over_ranks(total_ms, device=dev)
    ms_per_step = total_ms / args.steps
    value = cells * world * args.steps / (total_ms * 1e-3) / 1e9

    peak, peak_kind = hbm_peak()
    build_avg = statistics.mean(build_ms)
    trav_avg = statistics.mean(trav_ms)
    out_bytes = 32 * nverts
    alg_bytes = field_bytes + out_bytes
    gbs = lambda nbytes, ms: nbytes / (ms * 1e-3) / 1e9  # noqa: E731
    roof = {"kernel": "whole extraction step = classify_columns + reduce_levels + traverse_kernel "
                      "(three programmatically dependent launches)",
            "bound": "hbm", "achieved": gbs(alg_bytes, ms_per_step), "peak": peak, "unit": "GB/s",
            "frac": gbs(alg_bytes, ms_per_step) / peak,
            "traffic": BUILD_TRAFFIC_PER_FIELD_BYTE * field_bytes + TRAVERSE_TRAFFIC_PER_VERTEX * nverts,
            "traffic_source": "ncu dram__bytes_read+write of the 384^3 captures of the three kernels, scaled by "
                              "field bytes (build) and vertices (traversal)",
            "peak_kind": peak_kind, "algorithmic_bytes_per_launch": alg_bytes,
            "algorithmic_bytes": "field bytes read once + 32 B per vertex (float4 position + float4 normal)",
            "avg_launch_ms": ms_per_step,
            "timing": "CUDA events at the ends of K back-to-back steps on the launching stream",
            "frac_of_nominal": gbs(alg_bytes, ms_per_step) / NOMINAL_HBM_GBS}
    kernels = {
        "build": {"kernels": "classify_columns + reduce_levels", "ms": build_avg,
                  "algorithmic_bytes": field_bytes, "achieved_gbs": gbs(field_bytes, build_avg),
                  "frac": gbs(field_bytes, build_avg) / peak,
                  "traffic": BUILD_TRAFFIC_PER_FIELD_BYTE * field_bytes},
        "traverse": {"kernels": "traverse_kernel", "ms": trav_avg, "algorithmic_bytes": out_bytes,
                     "achieved_gbs": gbs(out_bytes, trav_avg), "frac": gbs(out_bytes, trav_avg) / peak,
                     "traffic": TRAVERSE_TRAFFIC_PER_VERTEX * nverts},
        "timing": "CUDA events around every build and extraction of a second pass of K steps",
    }
    step_frac = alg_bytes / (ms_per_step * 1e-3) / 1e9 / peak

    # --- e2e through the public API with host buffers ----------------------
    # Every step copies its field from pinned host memory, builds, reads the
    # count on the host, extracts and copies every vertex back.  Serial: one
    # volume at a time.  Pipelined (the reported value): two handles on two
    # streams, so the H2D copy of volume k+1 runs while volume k is built,
    # extracted and copied back (PCIe is full duplex).
    e2e = None
    if not args.no_e2e:
        h_field = torch.from_numpy(field_np).pin_memory()
        e2e_steps = max(4, min(args.steps, 10))

        class Slot:
            pass

        slots = []
        for k in range(2):
            sl = Slot()
            sl.h_pos = torch.empty((nverts, 4), dtype=torch.float32).pin_memory()
            sl.h_nrm = torch.empty((nverts, 4), dtype=torch.float32).pin_memory()
            if k == 0:
                sl.stream, sl.hp, sl.th, sl.field, sl.pos, sl.nrm = stream, hp, th, field, pos, nrm
            else:
                sl.stream = torch.cuda.Stream(device=dev)
                sl.field = torch.empty_like(field)
                sl.hp = H.HistoPyramid(C)
                sl.hp.set_stream(sl.stream)
                sl.hp.set_field_device(sl.field)
                sl.hp.set_normal_mode(H.NORMALS_CENTRAL)
                sl.th = H.TraversalHandle(sl.hp)
                sl.pos = torch.empty_like(pos)
                sl.nrm = torch.empty_like(nrm)
                sl.th.set_buffers(sl.pos, sl.nrm, nverts)
            slots.append(sl)
        counts = []

        def issue_in(k):  # H2D + build of volume k
            sl = slots[k % 2]
            with torch.cuda.stream(sl.stream):
                sl.field.copy_(h_field, non_blocking=True)
            sl.hp.build(iso)

        def finish(k):  # count (host sync), extraction, D2H of volume k
            sl = slots[k % 2]
            n = sl.hp.acquire_number_of_vertices()
            counts.append(n)
            sl.th.extract()
            with torch.cuda.stream(sl.stream):
                sl.h_pos[:n].copy_(sl.pos[:n], non_blocking=True)
                sl.h_nrm[:n].copy_(sl.nrm[:n], non_blocking=True)

        def serial(steps):
            for k in range(steps):
                issue_in(0)
                finish(0)

        def pipelined(steps):
            issue_in(0)
            for k in range(steps):
                if k + 1 < steps:
                    issue_in(k + 1)
                finish(k)

        def timed(fn, steps):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            slots[1].stream.wait_event(e0)
            fn(steps)
            stream.wait_stream(slots[1].stream)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / steps

        serial(2)  # warm-up of both legs
        pipelined(3)
        serial_ms = timed(serial, e2e_steps)
        e2e_ms = timed(pipelined, e2e_steps)
        assert all(n == nverts for n in counts), counts
        assert torch.equal(slots[0].h_pos[:nverts], slots[1].h_pos[:nverts])
        serial_ms = multi.max_over_ranks(serial_ms, device=dev)
        e2e_ms = multi.max_over_ranks(e2e_ms, device=dev)
        e2e = {"value": cells * world / (e2e_ms * 1e-3) / 1e9, "unit": "Gcells/s", "h2d_bytes_per_step": field_bytes,
               "d2h_bytes_per_step": 32 * nverts, "ms_per_step": e2e_ms, "volumes_in_flight": 2,
               "serial_value": cells * world / (serial_ms * 1e-3) / 1e9, "serial_ms_per_step": serial_ms}
        del slots

    batched = None
    if not args.no_batch:
        batched = run_batched(args, dev, stream, rank, world)
    adjoint = None
    if not args.no_adjoint:
        adjoint = run_adjoint(args, dev, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(field_np, iso, max_vertices=max(nverts, 1))

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Gcells/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32",
                "data": "synthetic: seeded Cayley cubic + N(0,1e-3) noise, generated in FP64, stored FP32",
                "config": {"workload": WORKLOAD if args.lattice == 512 else WORKLOAD.replace("512^3", f"{fx}^3"),
                           "lattice": [fx, fy, fz], "cells": cells, "vertices": nverts,
                           "classify_path": "tma_column" if path == 1 else "generic",
                           "normals": "central", "l2": "inputs larger than L2 (537 MB field per step)",
                           "parallelism": f"replicas x{world} (independent volumes)"},
                "roofline": roof,
                "kernels": kernels,
                "forward_normals_step_ms": fwd_ms,
                "forward_normals_value": cells * world / (fwd_ms * 1e-3) / 1e9,
                "step_hbm_fraction": step_frac,
                "step_hbm_fraction_of_nominal": alg_bytes / (ms_per_step * 1e-3) / 1e9 / NOMINAL_HBM_GBS,
                "step_algorithmic_bytes": alg_bytes,
                "vertices_per_s": nverts * world * args.steps / (total_ms * 1e-3),
                "build_ms": build_avg, "traverse_ms": trav_avg,
                "cpu_baseline": cpu, "e2e": e2e,
                "batched": batched,
                "adjoint": adjoint,
                "gpu_launches": 3 * args.steps,
                "gpu_launches_note": "classify + reduce + traverse per timed step (headline loop)",
                "clocks": clocks.summary()}
        print(json.dumps(line), flush=True)
    th.close()
    hp.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="hpmc", choices=["hpmc", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--lattice", type=int, default=512, help="lattice edge (profiling runs use smaller ones)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-extraction leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiable-extraction leg")
    ap.add_argument("--batch-tuning", default="",
                    help="fixed batch tuning 'column_slices,ctas_per_sm,rounds' instead of the autotuner "
                         "(profiling runs)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_hpmc(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
