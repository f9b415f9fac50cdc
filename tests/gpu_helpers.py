"""Helpers shared by the GPU tests: run the product through its C ABI and
compare with the oracle."""
from __future__ import annotations

import numpy as np

EPS32 = np.finfo(np.float32).eps


def run_gpu(hpmc, field, iso, *, cells=None, extent=(1.0, 1.0, 1.0), binary=False, unorm=False,
            normals=0, capture_codes=True, pitch_pad=0, tensor=None, gradient=False, texture=False):
    """Build + count + extract through the C ABI.  Returns a dict of numpy arrays.
    `field` is a numpy array ((z, y, x), or (z, y, x, 4) float32 gradient +
    value) or an oracle Functor (registered device functor).  texture=True
    (implied by gradient on an array) binds the array the reference's way:
    HPMCregisterDeviceField + HPMCsetFieldTexture3D(name, gradient)."""
    import torch

    dev = torch.device("cuda:0")
    fz, fy, fx = field.shape[:3]
    functor = hasattr(field, "params")
    if functor:
        pass
    elif tensor is None:
        if pitch_pad:
            big = torch.zeros((fz, fy, fx + pitch_pad), dtype=torch.from_numpy(field).dtype, device=dev)
            big[:, :, :fx] = torch.from_numpy(field).to(dev)
            tensor = big[:, :, :fx]
        else:
            tensor = torch.from_numpy(np.ascontiguousarray(field)).to(dev)
    c = hpmc.default_constants()
    hp = hpmc.HistoPyramid(c)
    hp.set_stream(torch.cuda.current_stream())
    name = None
    if functor:
        hp.set_lattice_size(fx, fy, fz)
        hp.set_field_custom(field.name, gradient=gradient)
        assert hp.builder_program() != 0
        if field.params:
            hp.set_builder_uniforms(field.params)
    elif texture or gradient:
        hp.set_lattice_size(fx, fy, fz)
        name = hpmc.register_device_field(tensor, unorm=unorm)
        hp.set_field_texture3d(name, gradient=gradient)
    else:
        hp.set_field_device(tensor, unorm=unorm)
    if cells is not None:
        hp.set_grid_size(*cells)
    hp.set_grid_extent(*extent)
    if binary:
        hp.set_field_as_binary()
    hp.set_normal_mode(normals)
    L = hp.layout()
    ncells = (cells if cells is not None else (fx - 1, fy - 1, fz - 1))
    codes_t = None
    if capture_codes:
        codes_t = torch.full((ncells[2], ncells[1], ncells[0]), 0xAB, dtype=torch.uint8, device=dev)
        hp.set_code_capture(codes_t)
    hp.build(iso)
    n = hp.acquire_number_of_vertices()
    assert hp.last_error == 0, hp.last_error
    path = hp.classify_path()
    levels = {}
    jtop = max(5, L[4] + 1)
    for j in range(5, jtop + 1):
        levels[j] = hp.read_level(j)
    th = hpmc.TraversalHandle(hp)
    m = max(n, 1)
    pos = torch.full((m, 4), float("nan"), dtype=torch.float32, device=dev)
    nrm = torch.full((m, 4), float("nan"), dtype=torch.float32, device=dev)
    info = torch.full((m, 4), -1, dtype=torch.int32, device=dev)
    tt = torch.full((m,), float("nan"), dtype=torch.float32, device=dev)
    th.set_debug_buffers(info, tt)
    written = th.extract_to(pos, nrm, n)
    status = hp.device_status()
    torch.cuda.synchronize()
    out = dict(n=n, written=written, layout=L, levels=levels, status=status, path=path,
               pos=pos[:n].cpu().numpy(), nrm=nrm[:n].cpu().numpy(), info=info[:n].cpu().numpy(),
               t=tt[:n].cpu().numpy())
    if capture_codes:
        out["codes"] = codes_t.cpu().numpy()
    th.close()
    hp.close()
    if name is not None:
        hpmc.unregister_device_field(name)
    return out


def oracle_expect(O, field, iso, *, cells=None, extent=(1.0, 1.0, 1.0), binary=False, unorm=False, normals=0):
    fz, fy, fx = field.shape[:3]
    L = O.layout((fx, fy, fz), cells)
    codes = O.codes(field, L, iso, binary=binary, unorm=unorm)
    levels, total = O.pyramid(codes, L)
    cell, code, k, edge = O.traverse(codes, levels, L, 0, total)
    t, pos, nrm = O.geometry(field, L, iso, cell, code, k, edge, binary=binary, normal_mode=normals,
                             extent=extent, unorm=unorm)
    return dict(L=L, codes=codes, levels=levels, total=total, cell=cell, code=code, k=k, edge=edge, t=t,
                pos=pos, nrm=nrm)


def angle(a, b):
    """Angle in radians between rows of a and b (float64)."""
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    na = np.linalg.norm(a, axis=1)
    nb = np.linalg.norm(b, axis=1)
    cross = np.linalg.norm(np.cross(a, b), axis=1)
    dot = (a * b).sum(1)
    return np.arctan2(cross, dot), na, nb


def compare(g, e, *, extent=(1.0, 1.0, 1.0), binary=False, check_geometry=True, normal_tol=1e-5):
    """Bit-exact topology, tolerance geometry.  Returns a small report dict."""
    L = e["L"]
    assert tuple(g["layout"]) == L.tile + L.layout + (L.size_l2, L.size)
    if "codes" in g:
        assert np.array_equal(g["codes"], e["codes"]), "case indices differ"
    for j, lv in g["levels"].items():
        if j <= L.size_l2 + 1:
            assert np.array_equal(lv, e["levels"][j]), f"pyramid level {j} differs"
        else:
            assert lv[0] == e["total"]
    assert g["n"] == e["total"], (g["n"], e["total"])
    assert g["written"] == e["total"]
    n = e["total"]
    info = g["info"]
    assert np.array_equal(info[:, :3], e["cell"]), "vertex -> cell order differs"
    assert np.array_equal(info[:, 3] & 0xff, e["code"].astype(np.int32))
    assert np.array_equal((info[:, 3] >> 8) & 0xff, e["k"].astype(np.int32))
    assert np.array_equal((info[:, 3] >> 16) & 0xff, e["edge"].astype(np.int32)), "vertex -> edge differs"
    rep = {"n": int(n)}
    if not check_geometry or n == 0:
        return rep
    spacing = np.array(extent, np.float64) / np.array(L.cells, np.float64)
    if not binary:
        dt = np.abs(g["t"].astype(np.float64) - e["t"])
        rep["max_dt"] = float(dt.max())
        assert rep["max_dt"] <= 1e-5, f"edge parameter t off by {rep['max_dt']}"
    # positions: 1e-5 of the lattice spacing on t plus FP32 rounding of the world coordinate
    dp = np.abs(g["pos"][:, :3].astype(np.float64) - e["pos"])
    tol = 1e-5 * spacing[None, :] + 4 * EPS32 * np.abs(e["pos"]) + 1e-30
    rep["max_pos_err_spacing"] = float((dp / spacing[None, :]).max())
    assert (dp <= tol).all(), f"position error {rep['max_pos_err_spacing']} spacings"
    assert np.all(g["pos"][:, 3] == 1.0)
    ang, na, nb = angle(g["nrm"][:, :3], e["nrm"])
    ok = nb > 1e-6 * max(1.0, float(nb.max()))
    rep["max_normal_angle"] = float(ang[ok].max()) if ok.any() else 0.0
    assert rep["max_normal_angle"] <= normal_tol, f"normal angle {rep['max_normal_angle']}"
    return rep
