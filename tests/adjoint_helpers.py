"""FP64 central finite differences of the extraction loss
L = sum_v dpos_v . p_v + dnrm_v . n_v with respect to single lattice samples,
for perturbations that keep every cell's case fixed (topology piecewise
constant).  Only the vertices whose stencil reads the perturbed sample are
re-evaluated; the others do not depend on it."""
from __future__ import annotations

import numpy as np


def stencil_index(field_shape, cell, edge, edge_table, central: bool):
    """Flat (z, y, x) indices of the samples each vertex reads, (n, 14) (clamped)."""
    fz, fy, fx = field_shape
    et = np.asarray(edge_table, np.float64)[edge]          # (n, 4): shift xyz, axis
    a = cell.astype(np.int64) + et[:, :3].astype(np.int64)
    axis = et[:, 3].astype(np.int64)
    b = a.copy()
    b[np.arange(len(b)), axis] += 1
    pts = [a, b]
    for i in range(3):
        e = np.zeros(3, np.int64)
        e[i] = 1
        pts += [a + e, b + e]
        if central:
            pts += [a - e, b - e]
    P = np.stack(pts, 1)                                    # (n, k, 3) as (x, y, z)
    P[..., 0] = np.clip(P[..., 0], 0, fx - 1)
    P[..., 1] = np.clip(P[..., 1], 0, fy - 1)
    P[..., 2] = np.clip(P[..., 2], 0, fz - 1)
    return (P[..., 2] * fy + P[..., 1]) * fx + P[..., 0]


def choose_samples(O, field, iso, cell, edge, count, seed, h, central):
    """Up to `count` samples (flat indices) read by at least one vertex whose
    perturbation by +-h keeps them on their side of iso (every case fixed);
    returns [(sample, vertex indices reading it)]."""
    idx = stencil_index(field.shape, cell, edge, O.edge_table(), central)
    flat = field.reshape(-1).astype(np.float64)
    order = np.argsort(idx, axis=None, kind="stable")
    keys = idx.reshape(-1)[order]
    verts = order // idx.shape[1]
    uniq, start = np.unique(keys, return_index=True)
    ends = np.append(start[1:], len(keys))
    cand = np.nonzero(np.abs(flat[uniq] - iso) > 2 * h)[0]
    rng = np.random.default_rng(seed)
    pick = rng.choice(cand, size=min(count, len(cand)), replace=False)
    return [(int(uniq[p]), np.unique(verts[start[p]:ends[p]])) for p in pick]


def fd_gradients(O, field, L, iso, cell, code, k, edge, dpos, dnrm, normal_mode, extent, samples, h):
    """FP64 central differences dL/df at each (sample, vertices) pair."""
    f64 = np.ascontiguousarray(field, dtype=np.float64)
    flat = f64.reshape(-1)
    out = np.zeros(len(samples))
    for j, (s, vs) in enumerate(samples):
        c, cd, kk, ee = cell[vs], code[vs], k[vs], edge[vs]
        dp, dn = dpos[vs], dnrm[vs]
        old = flat[s]
        vals = []
        for sgn in (1.0, -1.0):
            flat[s] = old + sgn * h
            _, p, n = O.geometry(f64, L, iso, c, cd, kk, ee, normal_mode=normal_mode, extent=extent)
            vals.append(float((dp * p).sum() + (dn * n).sum()))
        flat[s] = old
        out[j] = (vals[0] - vals[1]) / (2 * h)
    return out
