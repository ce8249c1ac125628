"""Mesh files (cupcfd_gpu_mesh_save / cupcfd_gpu_mesh_load).

The format is restated here in numpy (``mesh_file_bytes``) from its
description in include/cupcfd_gpu.h. CPU tests check that the library's
reader accepts the restatement's files and rejects every kind of damage
(wrong magic, version, header counts, flags, size, truncation, a flipped
byte) with the reference's error codes (E_FILE_MISSING, Error.h:44;
E_INVALID_FILE_FORMAT, Error.h:139) before any device work. GPU tests check
that the library writes the same bytes as the restatement, and that a
reloaded mesh gives bit-identical geometry, numbering, face-loop,
gradient, adjoint and boundary-loop results, in the same and in another
cell order.
"""
import ctypes as C
import os
import struct

import numpy as np
import pytest

import oracle as O
from test_oracle_vs_reference import _with_regions


def _fnv1a64(data: bytes) -> int:
    """FNV-1a over little-endian 64-bit words, a last partial word padded
    with zero bytes."""
    a = np.frombuffer(data + bytes(-len(data) % 8), "<u8")
    h = 1469598103934665603
    for w in a.tolist():
        h = ((h ^ w) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def mesh_file_bytes(m, splvl, rlencos=None, bnd_dist=None):
    """Bytes of a mesh file for the host mesh ``m`` (oracle dict, regions
    optional), split levels ``splvl`` and the optional momentum-loop
    geometry (rlencos per face, distance per boundary)."""
    nC, nF, nB = int(m["nCells"]), int(m["nFaces"]), int(m["nBnd"])
    nR = int(m.get("nRegions", 1))
    rtype = np.asarray(m.get("regionType", np.zeros(1, np.int32)), np.int32)
    ruvw = np.asarray(m.get("regionUVW", np.zeros(3)), np.float64).reshape(-1)
    rden = np.asarray(m.get("regionDen", np.zeros(1)), np.float64)
    breg = np.asarray(m.get("bndRegion", np.zeros(nB, np.int32)), np.int32)
    xp = np.asarray(m.get("faceXpac", np.zeros((nF, 3))), np.float64)
    xn = np.asarray(m.get("faceXnac", np.zeros((nF, 3))), np.float64)
    flags = int(bool(np.any(xp != 0) or np.any(xn != 0))) | (2 if rlencos is not None else 0) | \
        (4 if bnd_dist is not None else 0)
    hdr = b"CUPCFDM1" + struct.pack("<6i", 2, nC, nF, nB, nR, flags) + bytes(32)
    parts = [hdr]
    for k in ("faceCell1", "faceCell2", "faceBnd"):
        parts.append(np.ascontiguousarray(m[k], "<i4").tobytes())
    for k in ("faceLambda", "faceArea", "faceNorm", "faceCenter"):
        parts.append(np.ascontiguousarray(m[k], "<f8").tobytes())
    if flags & 1:
        parts += [np.ascontiguousarray(xp, "<f8").tobytes(), np.ascontiguousarray(xn, "<f8").tobytes()]
    parts += [np.ascontiguousarray(m["cellCenter"], "<f8").tobytes(), np.ascontiguousarray(m["cellVolume"], "<f8").tobytes(),
              rtype.astype("<i4").tobytes(), ruvw.astype("<f8").tobytes(), rden.astype("<f8").tobytes(),
              np.asarray(splvl, "<f8").tobytes(), breg.astype("<i4").tobytes()]
    if rlencos is not None:
        parts.append(np.ascontiguousarray(rlencos, "<f8").tobytes())
    if bnd_dist is not None:
        parts.append(np.ascontiguousarray(bnd_dist, "<f8").tobytes())
    body = b"".join(parts)
    return body + struct.pack("<Q", _fnv1a64(body))


def _case(xpac):
    m, splvl, rng = _with_regions(O.jitter(7, 6, 5, 0.25, seed=21, permute=True), 51)
    if xpac:
        m["faceXpac"] = rng.standard_normal((m["nFaces"], 3)) * 1e-3
        m["faceXnac"] = rng.standard_normal((m["nFaces"], 3)) * 1e-3
    return m, splvl


def _load_rc(cg, path):
    h = C.c_void_p()
    o = cg.MeshOptions(cg.ORDER_MORTON, (1 << cg.PREC_F64) | (1 << cg.PREC_F32C), -1)
    rc = cg.lib().cupcfd_gpu_mesh_load(os.fsencode(str(path)), C.byref(o), C.byref(h))
    if rc == cg.E_SUCCESS:
        cg.lib().cupcfd_gpu_mesh_destroy(h)
    return rc, cg.last_error()


# ---------------------------------------------------------------------------
# CPU: argument and file checks (all happen before device work)
# ---------------------------------------------------------------------------
def test_null_arguments(cg):
    L = cg.lib()
    h = C.c_void_p()
    assert L.cupcfd_gpu_mesh_save(None, b"x") == cg.E_NULL_PTR
    assert L.cupcfd_gpu_mesh_load(None, None, C.byref(h)) == cg.E_NULL_PTR
    assert L.cupcfd_gpu_mesh_load(b"x", None, None) == cg.E_NULL_PTR


def test_missing_file(cg, tmp_path):
    rc, msg = _load_rc(cg, tmp_path / "absent.cupcfdm")
    assert rc == cg.E_FILE_MISSING and "cannot open" in msg


@pytest.mark.parametrize("xpac,geom", [(False, False), (True, False), (False, True)])
def test_damaged_files_rejected(cg, tmp_path, xpac, geom):
    m, splvl = _case(xpac)
    rng = np.random.default_rng(5)
    rl, bd = (rng.uniform(0.1, 1, m["nFaces"]), rng.uniform(0.01, 0.1, m["nBnd"])) if geom else (None, None)
    good = mesh_file_bytes(m, splvl, rl, bd)
    p = tmp_path / "m.cupcfdm"

    def rc_of(data):
        p.write_bytes(data)
        return _load_rc(cg, p)

    bad = {
        "magic": b"CUPCFDM2" + good[8:],
        "version": good[:8] + struct.pack("<i", 3) + good[12:],
        "cells0": good[:12] + struct.pack("<i", 0) + good[16:],
        "faces+1": good[:16] + struct.pack("<i", int(m["nFaces"]) + 1) + good[20:],
        "flags": good[:28] + struct.pack("<i", 8) + good[32:],
        "flags without arrays": good[:28] + struct.pack("<i", 6 | (1 if xpac else 0)) + good[32:] if not geom else
        good[:28] + struct.pack("<i", 1 if xpac else 0) + good[32:],
        "truncated": good[:-9],
        "extra": good + b"\0",
        "header only": good[:64],
        "empty": b"",
    }
    for what, data in bad.items():
        rc, msg = rc_of(data)
        assert rc == cg.E_INVALID_FILE_FORMAT, (what, rc, msg)
    for off in (64, len(good) // 2, len(good) - 9, len(good) - 1):   # first array byte, middle, last array byte, hash
        data = bytearray(good)
        data[off] ^= 0x10
        rc, msg = rc_of(bytes(data))
        assert rc == cg.E_INVALID_FILE_FORMAT and ("checksum" in msg), (off, rc, msg)
    # the intact file passes every format check (without a GPU, mesh
    # creation is what fails, with another code)
    rc, msg = rc_of(good)
    assert rc not in (cg.E_FILE_MISSING, cg.E_INVALID_FILE_FORMAT), (rc, msg)


# ---------------------------------------------------------------------------
# GPU: round trips
# ---------------------------------------------------------------------------
def _forward_results(cg, mesh, ref, seed):
    f = O.fields(ref, seed)
    gface = np.random.Generator(np.random.Philox(key=seed + 1)).standard_normal(ref["nFaces"])
    r = {}
    for prec in (cg.PREC_F64, cg.PREC_F32C):
        # host FP64 buffers for both precisions; FP32-representable values for F32C
        cast = (lambda a: a) if prec == cg.PREC_F64 else (lambda a: a.astype(np.float32).astype(np.float64))
        out = cg.forward_adjoint(mesh, prec, cast(f["phi"]), cast(f["phiB"]), cast(f["den"]), cast(f["u"]),
                                 cast(f["v"]), cast(f["w"]), cast(gface))
        r.update({f"{prec}:{k}": v.copy() for k, v in out.items()})
    return r


def _face_loop_results(cg, mesh, ref, seed):
    from test_gpu_parity import _mass_case
    f = O.fields(ref, seed, full=True)
    f["massFlux"] = np.random.default_rng(seed).standard_normal(ref["nFaces"])
    f["solveTurbEnergy"] = f["solveEnthalpy"] = True
    rc, o = _mass_case(cg, mesh, ref, f)
    assert rc == cg.E_SUCCESS
    return o


def _assert_same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


@pytest.mark.gpu
@pytest.mark.parametrize("xpac", [False, True])
def test_save_writes_the_format(cg, gpu, tmp_path, xpac):
    m, splvl = _case(xpac)
    mesh = cg.Mesh.from_arrays(m, order=cg.ORDER_RCM)
    assert mesh.set_regions(m["regionType"], m["regionUVW"], m["regionDen"], m["bndRegion"]) == cg.E_SUCCESS
    assert mesh.set_region_split(splvl) == cg.E_SUCCESS
    p = tmp_path / "m.cupcfdm"
    assert mesh.save(p) == cg.E_SUCCESS
    assert p.read_bytes() == mesh_file_bytes(m, splvl)


@pytest.mark.gpu
@pytest.mark.parametrize("xpac", [False, True])
@pytest.mark.parametrize("order2", ["same", "other"])
def test_round_trip_bit_identical(cg, gpu, tmp_path, xpac, order2):
    from test_gpu_boundary_loops import _host_chain
    m, splvl = _case(xpac)
    order = cg.ORDER_MORTON
    mesh = cg.Mesh.from_arrays(m, order=order)
    assert mesh.set_regions(m["regionType"], m["regionUVW"], m["regionDen"], m["bndRegion"]) == cg.E_SUCCESS
    assert mesh.set_region_split(splvl) == cg.E_SUCCESS
    p = tmp_path / "m.cupcfdm"
    assert mesh.save(p) == cg.E_SUCCESS
    loaded = cg.Mesh.load(p, order=order if order2 == "same" else cg.ORDER_RCM)
    assert (loaded.nCells, loaded.nFaces, loaded.nBoundaries, loaded.nIncidences) == \
        (mesh.nCells, mesh.nFaces, mesh.nBoundaries, mesh.nIncidences)
    _assert_same(mesh.geometry(), loaded.geometry())
    _assert_same(dict(zip("xa", mesh.cell_face_csr())), dict(zip("xa", loaded.cell_face_csr())))
    if order2 == "same":
        _assert_same(dict(zip("cf", mesh.numbering())), dict(zip("cf", loaded.numbering())))
    a, b = _forward_results(cg, mesh, m, 61), _forward_results(cg, loaded, m, 61)
    if order2 == "other":
        # the loss is summed over faces in the layout's order: equal to rounding
        for k in [k for k in a if k.endswith(":loss")]:
            assert abs(a[k][0] - b.pop(k)[0]) <= 1e-12 * abs(a.pop(k)[0]), k
    _assert_same(a, b)
    _assert_same(_face_loop_results(cg, mesh, m, 62), _face_loop_results(cg, loaded, m, 62))
    rng = np.random.Generator(np.random.Philox(key=63))
    nF, nB, nC, nR = m["nFaces"], m["nBnd"], m["nCells"], m["nRegions"]
    d = dict(mf=rng.uniform(1e-6, 1e-2, nF) * rng.choice([-1.0, 1.0], nF),
             u=rng.uniform(1e-6, 1e-2, nB), v=rng.uniform(1e-6, 1e-2, nB), w=rng.uniform(1e-6, 1e-2, nB),
             den=rng.uniform(0.9, 1.1, nB), fr=rng.uniform(1e-6, 1e-2, nR), su=rng.standard_normal(nC))
    _assert_same(_host_chain(cg, mesh, d, (1, 1, 1)), _host_chain(cg, loaded, d, (1, 1, 1)))
    # a second save of the loaded mesh gives the same file
    p2 = tmp_path / "m2.cupcfdm"
    assert loaded.save(p2) == cg.E_SUCCESS
    assert p2.read_bytes() == p.read_bytes()


@pytest.mark.gpu
def test_structgen_mesh_round_trip(cg, gpu, tmp_path):
    """A mesh generated on the device (no host copy exists) saves and
    reloads; its file equals the restatement's file of the oracle's mesh
    (the device generator is bit-identical to the oracle's), with the
    single default region."""
    mesh = cg.Mesh.structgen(9, 8, 7)
    p = tmp_path / "s.cupcfdm"
    assert mesh.save(p) == cg.E_SUCCESS
    loaded = cg.Mesh.load(p)
    _assert_same(mesh.geometry(), loaded.geometry())
    assert p.read_bytes() == mesh_file_bytes(O.structgen(9, 8, 7), np.zeros(1))
    with pytest.raises(cg.CupcfdError):
        cg.Mesh.load(tmp_path / "absent.cupcfdm")


@pytest.mark.gpu
def test_round_trip_momentum_geometry(cg, gpu, tmp_path):
    """rlencos and boundary distances travel with the file, and the momentum
    loop gives the same bits on the loaded mesh."""
    from test_gpu_uvw import _host, _check
    from test_oracle_vs_reference import uvw_case
    m, rng = uvw_case("jitter", 80, "outlet")
    rl, bd = rng.uniform(0.1, 2.0, m["nFaces"]), rng.uniform(0.01, 0.2, m["nBnd"])
    mesh = cg.Mesh.from_arrays(m, order=cg.ORDER_MORTON)
    assert mesh.set_regions(m["regionType"], m["regionUVW"], m["regionDen"], m["bndRegion"]) == cg.E_SUCCESS
    assert mesh.set_face_rlencos(rl) == cg.E_SUCCESS and mesh.set_boundary_distance(bd) == cg.E_SUCCESS
    p = tmp_path / "g.cupcfdm"
    assert mesh.save(p) == cg.E_SUCCESS
    assert p.read_bytes() == mesh_file_bytes(m, np.zeros(m["nRegions"]), rl, bd)
    loaded = cg.Mesh.load(p, order=cg.ORDER_RCM)
    f = O.uvw_fields(m, 81)
    _check(_host(cg, loaded, f), O.uvw_face_loop1(m, f, rl, bd))
