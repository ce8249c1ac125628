"""ctypes front end of the test-only checkers.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, never by the CUDA library's own code.

* ``liboracle.so`` -- the plain-C restatement in cupcfd_oracle.c (always
  buildable: ``make -C oracle``).
* ``_ref/libcupcfd_ref.so`` -- the reference's own sources compiled unchanged
  (``make -C oracle ref``); present only where it was built from a reference
  source tree, so everything using it is optional.

Meshes are dicts of numpy arrays in the reference's local numbering
(faces, cells and boundaries in ascending label order); 3-vectors are
``(n, 3)`` float64 arrays.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lock = threading.Lock()
_lib = None
_ref = None
_ref_tried = False

E_SUCCESS = 95
E_INVALID_INDEX = 68
E_ARRAY_SIZE_MISMATCH = 25
E_ERROR = 98


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


def load():
    """Load (building on first use) the C restatement."""
    global _lib
    with _lock:
        if _lib is None:
            so = os.path.join(HERE, "liboracle.so")
            src = os.path.join(HERE, "cupcfd_oracle.c")
            if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
                subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
            _lib = C.CDLL(so)
            _lib.orc_jitter_build.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_ulonglong, C.c_int] + [C.c_void_p] * 11
            _lib.orc_structgen_build.argtypes = [C.c_int] * 3 + [C.c_double] * 6 + [C.c_void_p] * 11
            _lib.orc_flux_mass_face_loop.argtypes = [C.c_void_p] * 15 + [C.c_double] + [C.c_void_p] * 4 + [C.c_int] * 4 + [C.c_void_p] * 8
            _lib.orc_boundary_loop3.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
            _lib.orc_boundary_loop4.argtypes = [C.c_void_p] * 7 + [C.c_double, C.c_void_p]
            _lib.orc_boundary_loop5.argtypes = [C.c_void_p] * 6 + [C.c_double] + [C.c_int] * 3 + [C.c_void_p] * 2
            _lib.orc_region_loop.argtypes = [C.c_void_p] * 4 + [C.c_double]
            _lib.orc_uvw_face_loop1.argtypes = [C.c_void_p] * 3 + [C.c_double] * 2 + [C.c_void_p] * 20
        return _lib


def load_ref():
    """Load the reference build if it exists (None otherwise)."""
    global _ref, _ref_tried
    with _lock:
        if not _ref_tried:
            _ref_tried = True
            so = os.path.join(HERE, "_ref", "libcupcfd_ref.so")
            if os.path.exists(so):
                _ref = C.CDLL(so)
                _ref.ref_structgen_build.argtypes = [C.c_int] * 3 + [C.c_double] * 6 + [C.c_void_p] * 13
                _ref.ref_ctx_create.restype = C.c_void_p
                _ref.ref_ctx_create.argtypes = [C.c_int] * 4 + [C.c_void_p] * 15
                _ref.ref_ctx_destroy.argtypes = [C.c_void_p]
                _ref.ref_gradient_phi_gauss.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                                        C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
                _ref.ref_flux_mass_face_loop.argtypes = ([C.c_void_p] * 15 + [C.c_double] + [C.c_void_p] * 4
                                                         + [C.c_int] * 4 + [C.c_void_p] * 8 + [C.c_int, C.c_void_p])
                _ref.ref_ctx_set_splvl.argtypes = [C.c_void_p, C.c_void_p]
                _ref.ref_boundary_loop1.argtypes = [C.c_void_p] * 3
                _ref.ref_boundary_loop2.argtypes = [C.c_void_p] * 4
                _ref.ref_boundary_loop3.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
                _ref.ref_boundary_loop4.argtypes = [C.c_void_p] * 6 + [C.c_double, C.c_void_p]
                _ref.ref_boundary_loop5.argtypes = [C.c_void_p] * 6 + [C.c_double] + [C.c_int] * 3 + [C.c_void_p] * 2
                _ref.ref_region_loop.argtypes = [C.c_void_p] * 3 + [C.c_double]
                _ref.ref_boundary_chain.argtypes = [C.c_void_p] * 9 + [C.c_int, C.c_void_p]
                _ref.ref_gradient_phi_gauss_f32.argtypes = [C.c_int] * 3 + [C.c_void_p] * 8 + [C.c_int] + [C.c_void_p] * 4
                _ref.ref_ctx_set_uvw_geometry.argtypes = [C.c_void_p] * 3
                _ref.ref_uvw_state.argtypes = [C.c_void_p] * 5
                _ref.ref_uvw_face_loop1.argtypes = [C.c_void_p, C.c_double, C.c_double] + [C.c_void_p] * 19 + [C.c_int, C.c_void_p]
                _ref.ref_uvw_region_loop1.argtypes = [C.c_void_p]
                _ref.ref_uvw_bnds_loop1.argtypes = [C.c_void_p]
        return _ref


def ref_gradient_f32(m, phi, phiB, nGradient):
    """GradientPhiGaussDolfyn of the reference's T=float instantiation
    (compiled unchanged) on mesh ``m`` with its geometry rounded to float:
    (dPhidx, dPhidxo) as float32 [nCells, 3]."""
    ref = load_ref()
    assert ref is not None, "reference build absent"
    f32 = lambda k: np.ascontiguousarray(np.asarray(m[k]).reshape(-1), np.float32)
    i32 = lambda k: np.ascontiguousarray(m[k], np.int32)
    nC, nF, nB = int(m["nCells"]), int(m["nFaces"]), int(m["nBnd"])
    g, go = np.zeros((nC, 3), np.float32), np.zeros((nC, 3), np.float32)
    a = [i32("faceCell1"), i32("faceCell2"), i32("faceBnd"), f32("faceLambda"), f32("faceNorm"), f32("faceCenter"),
         f32("cellCenter"), f32("cellVolume")]
    ph, pb = np.ascontiguousarray(phi, np.float32), np.ascontiguousarray(phiB, np.float32)
    rc = ref.ref_gradient_phi_gauss_f32(nC, nF, nB, *[_p(x) for x in a], int(nGradient), _p(ph), _p(pb), _p(g), _p(go))
    assert rc == E_SUCCESS, rc
    return g, go


def ref_flux_mass_f32(m, f):
    """FluxMassDolfynFaceLoop of the reference's T=float instantiation
    (compiled unchanged) on mesh ``m`` with its geometry and regions rounded
    to float, fields ``f`` (as fields(full=True)) rounded to float. Returns
    (rc, out) like flux_mass_face_loop, out arrays float32."""
    ref = load_ref()
    assert ref is not None, "reference build absent"
    f32 = lambda x: np.ascontiguousarray(np.asarray(x).reshape(-1), np.float32)
    i32 = lambda x: np.ascontiguousarray(x, np.int32)
    nC, nF, nB, nR = int(m["nCells"]), int(m["nFaces"]), int(m["nBnd"]), int(m["nRegions"])
    geo = [i32(m["faceCell1"]), i32(m["faceCell2"]), i32(m["faceBnd"])] + [
        f32(m[k]) for k in ("faceLambda", "faceNorm", "faceCenter", "faceArea", "faceXpac", "faceXnac", "cellCenter",
                            "cellVolume")] + [i32(m["bndRegion"]), i32(m["regionType"]), f32(m["regionUVW"]), f32(m["regionDen"])]
    a = {k: f32(f[k]) for k in ("dudx", "dvdx", "dwdx", "dpdx", "den", "u", "v", "w", "p", "ar", "teC", "edC", "visC", "tC")}
    out = {k: f32(f[k]).copy() for k in ("massFlux", "su", "rface", "denB", "teB", "edB", "visB", "tB")}
    cnt = [C.c_int(int(f.get(k, 0))) for k in ("icinl", "icout", "icsym", "icwal")]
    fn = ref.ref_flux_mass_face_loop_f32
    fn.argtypes = [C.c_int] * 4 + [C.c_void_p] * 29 + [C.c_float] + [C.c_void_p] * 4 + [C.c_int] * 4 + [C.c_void_p] * 8
    rc = fn(nC, nF, nB, nR, *[_p(x) for x in geo], _p(a["dudx"]), _p(a["dvdx"]), _p(a["dwdx"]), _p(a["dpdx"]),
            _p(a["den"]), _p(out["denB"]), _p(a["u"]), _p(a["v"]), _p(a["w"]), _p(out["massFlux"]), _p(a["p"]),
            _p(a["ar"]), _p(out["su"]), _p(out["rface"]), float(np.float32(f["small"])), *[C.byref(c) for c in cnt],
            *[int(bool(f.get(k, False))) for k in ("solveTurbEnergy", "solveTurbDiss", "solveVisc", "solveEnthalpy")],
            _p(a["teC"]), _p(out["teB"]), _p(a["edC"]), _p(out["edB"]), _p(a["visC"]), _p(out["visB"]), _p(a["tC"]),
            _p(out["tB"]))
    out.update(icinl=cnt[0].value, icout=cnt[1].value, icsym=cnt[2].value, icwal=cnt[3].value)
    return rc, out


# ---------------------------------------------------------------------------
# meshes
# ---------------------------------------------------------------------------

def counts(nx, ny, nz):
    nc = nx * ny * nz
    nf = ny * nz * (nx + 1) + nx * nz * (ny + 1) + nx * ny * (nz + 1)
    nb = 2 * (ny * nz + nx * nz + nx * ny)
    nv = (nx + 1) * (ny + 1) * (nz + 1)
    return nc, nf, nb, nv


def _alloc_mesh(nc, nf, nb):
    return dict(
        nCells=nc, nFaces=nf, nBnd=nb,
        faceCell1=np.empty(nf, np.int32), faceCell2=np.empty(nf, np.int32), faceBnd=np.empty(nf, np.int32),
        faceLambda=np.empty(nf), faceNorm=np.empty((nf, 3)), faceCenter=np.empty((nf, 3)), faceArea=np.empty(nf),
        cellCenter=np.empty((nc, 3)), cellVolume=np.empty(nc),
    )


def _finish_mesh(m):
    nf, nb = m["nFaces"], m["nBnd"]
    m["faceXpac"] = np.zeros((nf, 3))            # addData passes xpac = xnac = 0 (UnstructuredMeshInterface.ipp:1778-1780)
    m["faceXnac"] = np.zeros((nf, 3))
    m["nRegions"] = 1
    m["bndRegion"] = np.zeros(nb, np.int32)      # one region, label 0
    m["regionType"] = np.zeros(1, np.int32)      # RTYPE_DEFAULT (CupCfdSoAMesh.cpp:211-221)
    m["regionUVW"] = np.zeros((1, 3))
    m["regionDen"] = np.zeros(1)
    return m


def structgen(nx, ny, nz, bounds=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), with_vertices=False):
    """Structured hex mesh from the C restatement of MeshStructGenSource."""
    nc, nf, nb, nv = counts(nx, ny, nz)
    m = _alloc_mesh(nc, nf, nb)
    fv = np.empty((nf, 4), np.int32) if with_vertices else None
    vc = np.empty((nv, 3)) if with_vertices else None
    rc = load().orc_structgen_build(nx, ny, nz, *[float(b) for b in bounds],
                                    _p(m["faceCell1"]), _p(m["faceCell2"]), _p(m["faceBnd"]),
                                    _p(m["faceLambda"]), _p(m["faceNorm"]), _p(m["faceCenter"]), _p(m["faceArea"]),
                                    _p(m["cellCenter"]), _p(m["cellVolume"]), _p(fv), _p(vc))
    assert rc == E_SUCCESS, rc
    if with_vertices:
        m["faceVert"], m["vertCoords"] = fv, vc
    return _finish_mesh(m)


def structgen_cell_face_labels(nx, ny, nz):
    nc = nx * ny * nz
    xadj = np.empty(nc + 1, np.int32)
    adj = np.empty(6 * nc, np.int32)
    load().orc_structgen_cell_face_labels(nx, ny, nz, _p(xadj), _p(adj))
    return xadj, adj


def jitter(nx, ny, nz, amount=0.25, seed=1, permute=True):
    """Jittered, optionally permuted hex mesh (geometry defined in cupcfd_oracle.c)."""
    nc, nf, nb, _ = counts(nx, ny, nz)
    m = _alloc_mesh(nc, nf, nb)
    cp = np.empty(nc, np.int32)
    fp = np.empty(nf, np.int32)
    rc = load().orc_jitter_build(nx, ny, nz, float(amount), int(seed), int(bool(permute)),
                                 _p(m["faceCell1"]), _p(m["faceCell2"]), _p(m["faceBnd"]),
                                 _p(m["faceLambda"]), _p(m["faceNorm"]), _p(m["faceCenter"]), _p(m["faceArea"]),
                                 _p(m["cellCenter"]), _p(m["cellVolume"]), _p(cp), _p(fp))
    assert rc == E_SUCCESS, rc
    m["cellPerm"], m["facePerm"] = cp, fp
    return _finish_mesh(m)


def merge_cells(m, frac=0.3, seed=1, max_cells=3):
    """A polyhedral mesh from a hex mesh: interior faces removed at random
    (a fraction ``frac`` of them, in a seeded order) with their two cells
    merged into one; a merged cell holds at most ``max_cells`` hexahedra
    (cells of 6 to 14 faces, more with a larger cap), so the cells of a
    32-cell slice have different face counts. The merged cell keeps its lowest label; cells are relabelled
    in ascending order, faces keep their relative order, boundaries their
    ids. Centre = mean of the merged centres, volume = their sum. Geometry is
    then not that of a real polyhedron, which the face loops do not need:
    they are checked for bit-identity on whatever arrays the mesh holds."""
    nc, nf = int(m["nCells"]), int(m["nFaces"])
    rng = np.random.Generator(np.random.Philox(key=seed))
    parent = np.arange(nc)

    def find(c):
        while parent[c] != c:
            parent[c] = parent[parent[c]]
            c = parent[c]
        return c

    c1, c2 = m["faceCell1"].astype(np.int64), m["faceCell2"].astype(np.int64)
    interior = np.flatnonzero(c2 >= 0)
    order = rng.permutation(interior)
    removed = np.zeros(nf, bool)
    size = np.ones(nc, np.int64)
    for f in order[: int(frac * len(interior))]:
        a, b = find(c1[f]), find(c2[f])
        if a == b or size[a] + size[b] > max_cells:
            continue
        lo, hi = min(a, b), max(a, b)
        parent[hi] = lo
        size[lo] += size[hi]
    rep = np.array([find(c) for c in range(nc)])
    # faces whose two cells now coincide disappear
    for f in interior:
        if rep[c1[f]] == rep[c2[f]]:
            removed[f] = True
    keep_cells = np.flatnonzero(rep == np.arange(nc))
    new_id = -np.ones(nc, np.int64)
    new_id[keep_cells] = np.arange(len(keep_cells))
    keep_f = np.flatnonzero(~removed)
    out = dict(m)
    out["nCells"], out["nFaces"] = int(len(keep_cells)), int(len(keep_f))
    out["faceCell1"] = new_id[rep[c1[keep_f]]].astype(np.int32)
    c2k = c2[keep_f]
    out["faceCell2"] = np.where(c2k >= 0, new_id[rep[np.maximum(c2k, 0)]], -1).astype(np.int32)
    for k in ("faceBnd", "faceLambda", "faceArea"):
        out[k] = np.ascontiguousarray(m[k][keep_f])
    for k in ("faceNorm", "faceCenter", "faceXpac", "faceXnac"):
        out[k] = np.ascontiguousarray(m[k][keep_f])
    cc = np.zeros((len(keep_cells), 3))
    cnt = np.zeros(len(keep_cells))
    vol = np.zeros(len(keep_cells))
    np.add.at(cc, new_id[rep], m["cellCenter"])
    np.add.at(cnt, new_id[rep], 1.0)
    np.add.at(vol, new_id[rep], m["cellVolume"])
    out["cellCenter"] = cc / cnt[:, None]
    out["cellVolume"] = vol
    for k in ("cellPerm", "facePerm"):
        out.pop(k, None)
    return out


def cell_face_csr(m):
    nc, nf = m["nCells"], m["nFaces"]
    nnz = int(nf + np.count_nonzero(m["faceCell2"] >= 0))
    xadj = np.empty(nc + 1, np.int32)
    adj = np.empty(nnz, np.int32)
    rc = load().orc_cell_face_csr(nc, nf, _p(m["faceCell1"]), _p(m["faceCell2"]), _p(xadj), _p(adj))
    assert rc == E_SUCCESS, rc
    return xadj, adj


class _OrcMesh(C.Structure):
    _fields_ = [("nCells", C.c_int), ("nFaces", C.c_int), ("nBnd", C.c_int), ("nRegions", C.c_int)] + [
        (n, C.c_void_p) for n in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceNorm", "faceCenter",
                                  "faceArea", "faceXpac", "faceXnac", "cellCenter", "cellVolume", "bndRegion",
                                  "regionType", "regionUVW", "regionDen")]


def _cmesh(m):
    s = _OrcMesh()
    for k in ("nCells", "nFaces", "nBnd", "nRegions"):
        setattr(s, k, int(m[k]))
    for k, _ in _OrcMesh._fields_[4:]:
        setattr(s, k, _p(m[k]).value if m[k] is not None else None)
    return s


# ---------------------------------------------------------------------------
# kernels (C restatement)
# ---------------------------------------------------------------------------

def gradient(m, phi, phib, n_gradient=1):
    nc = m["nCells"]
    g = np.empty((nc, 3))
    go = np.empty((nc, 3))
    s = _cmesh(m)
    phi = np.ascontiguousarray(phi, np.float64)
    phib = np.ascontiguousarray(phib, np.float64)
    rc = load().orc_gradient_phi_gauss(C.byref(s), n_gradient, _p(phi), len(phi), _p(phib), len(phib),
                                       _p(g), nc, _p(go), nc)
    return rc, g, go


def flux_mass_face_loop(m, f):
    """Full FluxMassDolfynFaceLoop. ``f`` is a dict of input arrays; the
    in/out arrays (massFlux, su, rface, denB, teB, edB, visB, tB) are copied
    and returned with the four counters."""
    out = {k: np.array(f[k], np.float64, copy=True) for k in ("massFlux", "su", "rface", "denB", "teB", "edB", "visB", "tB")}
    cnt = [C.c_int(int(f.get(k, 0))) for k in ("icinl", "icout", "icsym", "icwal")]
    s = _cmesh(m)
    a = {k: np.ascontiguousarray(f[k], np.float64) for k in ("dudx", "dvdx", "dwdx", "dpdx", "den", "u", "v", "w", "p", "ar",
                                                             "teC", "edC", "visC", "tC")}
    rc = load().orc_flux_mass_face_loop(
        C.byref(s), _p(a["dudx"]), _p(a["dvdx"]), _p(a["dwdx"]), _p(a["dpdx"]), _p(a["den"]), _p(out["denB"]),
        _p(a["u"]), _p(a["v"]), _p(a["w"]), _p(out["massFlux"]), _p(a["p"]), _p(a["ar"]), _p(out["su"]), _p(out["rface"]),
        float(f["small"]), *[C.byref(c) for c in cnt],
        *[int(bool(f.get(k, False))) for k in ("solveTurbEnergy", "solveTurbDiss", "solveVisc", "solveEnthalpy")],
        _p(a["teC"]), _p(out["teB"]), _p(a["edC"]), _p(out["edB"]), _p(a["visC"]), _p(out["visB"]), _p(a["tC"]), _p(out["tB"]))
    out.update(icinl=cnt[0].value, icout=cnt[1].value, icsym=cnt[2].value, icwal=cnt[3].value)
    return rc, out


def mass_plain(m, den, u, v, w, massflux_in=None):
    mf = np.zeros(m["nFaces"]) if massflux_in is None else np.array(massflux_in, np.float64, copy=True)
    s = _cmesh(m)
    args = [np.ascontiguousarray(x, np.float64) for x in (den, u, v, w)]
    rc = load().orc_mass_plain_forward(C.byref(s), *[_p(x) for x in args], _p(mf))
    assert rc == E_SUCCESS
    return mf


def mass_plain_adjoint(m, den, u, v, w, mbar):
    nc = m["nCells"]
    outs = [np.empty(nc) for _ in range(4)]
    s = _cmesh(m)
    args = [np.ascontiguousarray(x, np.float64) for x in (den, u, v, w, mbar)]
    rc = load().orc_mass_plain_adjoint(C.byref(s), *[_p(x) for x in args], *[_p(o) for o in outs])
    assert rc == E_SUCCESS
    return outs


def gradient_adjoint(m, gbar):
    phibar = np.empty(m["nCells"])
    phibbar = np.empty(m["nBnd"])
    s = _cmesh(m)
    gbar = np.ascontiguousarray(gbar, np.float64)
    rc = load().orc_gradient_adjoint(C.byref(s), _p(gbar), _p(phibar), _p(phibbar))
    assert rc == E_SUCCESS
    return phibar, phibbar


# ---------------------------------------------------------------------------
# boundary / region loops (C restatement of MassKernels.ipp:311-554). Each
# takes and returns copies: the in/out arrays of the reference call are
# returned updated, its scalar outputs as floats.
# ---------------------------------------------------------------------------
def _f64(a):
    return np.array(a, np.float64, copy=True)


def boundary_loop1(m, massflux):
    out = C.c_double(np.nan)
    mf = np.ascontiguousarray(massflux, np.float64)
    assert load().orc_boundary_loop1(C.byref(_cmesh(m)), _p(mf), C.byref(out)) == E_SUCCESS
    return out.value


def boundary_loop2(m, massflux, flow_region):
    out = C.c_double(np.nan)
    mf, fr = np.ascontiguousarray(massflux, np.float64), _f64(flow_region)
    assert load().orc_boundary_loop2(C.byref(_cmesh(m)), _p(mf), _p(fr), C.byref(out)) == E_SUCCESS
    return fr, out.value


def boundary_loop3(m, flowin):
    out = C.c_double(np.nan)
    assert load().orc_boundary_loop3(C.byref(_cmesh(m)), float(flowin), C.byref(out)) == E_SUCCESS
    return out.value


def boundary_loop4(m, splvl, massflux, ub, vb, wb, denb, ratearea):
    out = C.c_double(np.nan)
    mf, u, v, w = _f64(massflux), _f64(ub), _f64(vb), _f64(wb)
    sp, den = np.ascontiguousarray(splvl, np.float64), np.ascontiguousarray(denb, np.float64)
    assert load().orc_boundary_loop4(C.byref(_cmesh(m)), _p(sp), _p(mf), _p(u), _p(v), _p(w), _p(den), float(ratearea),
                                     C.byref(out)) == E_SUCCESS
    return mf, u, v, w, out.value


def boundary_loop5(m, massflux, su, ub, vb, wb, fact, solve, flow_fact, flowout2):
    out = C.c_double(flowout2)
    mf, s_, u, v, w = _f64(massflux), _f64(su), _f64(ub), _f64(vb), _f64(wb)
    ff = np.ascontiguousarray(flow_fact, np.float64)
    assert load().orc_boundary_loop5(C.byref(_cmesh(m)), _p(mf), _p(s_), _p(u), _p(v), _p(w), float(fact),
                                     *[int(bool(x)) for x in solve], _p(ff), C.byref(out)) == E_SUCCESS
    return mf, s_, u, v, w, out.value


def region_loop(m, splvl, flow_region, flow_in):
    ff = np.full(m["nRegions"], np.nan)
    sp, fr = np.ascontiguousarray(splvl, np.float64), np.ascontiguousarray(flow_region, np.float64)
    assert load().orc_region_loop(C.byref(_cmesh(m)), _p(sp), _p(ff), _p(fr), float(flow_in)) == E_SUCCESS
    return ff


# ---------------------------------------------------------------------------
# the reference's own code (optional)
# ---------------------------------------------------------------------------

def ref_structgen(nx, ny, nz, bounds=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), with_vertices=False):
    ref = load_ref()
    if ref is None:
        return None
    nc, nf, nb, nv = counts(nx, ny, nz)
    m = _alloc_mesh(nc, nf, nb)
    xadj = np.empty(nc + 1, np.int32)
    adj = np.empty(6 * nc, np.int32)
    fv = np.empty((nf, 4), np.int32) if with_vertices else None
    vc = np.empty((nv, 3)) if with_vertices else None
    rc = ref.ref_structgen_build(nx, ny, nz, *[float(b) for b in bounds],
                                 _p(m["faceCell1"]), _p(m["faceCell2"]), _p(m["faceBnd"]),
                                 _p(m["faceLambda"]), _p(m["faceNorm"]), _p(m["faceCenter"]), _p(m["faceArea"]),
                                 _p(m["cellCenter"]), _p(m["cellVolume"]), _p(xadj), _p(adj), _p(fv), _p(vc))
    assert rc == E_SUCCESS, rc
    m["srcCellFaceXAdj"], m["srcCellFaceAdj"] = xadj, adj
    if with_vertices:
        m["faceVert"], m["vertCoords"] = fv, vc
    return _finish_mesh(m)


class RefKernels:
    """The reference's GradientPhiGaussDolfyn / FluxMassDolfynFaceLoop over a
    mesh dict. Keeps references to the arrays it was given."""

    def __init__(self, m):
        self.ref = load_ref()
        if self.ref is None:
            raise RuntimeError("reference build absent (make -C oracle ref)")
        self.m = {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v) for k, v in m.items()}
        mm = self.m
        self.h = self.ref.ref_ctx_create(mm["nCells"], mm["nFaces"], mm["nBnd"], mm["nRegions"],
                                         *[_p(mm[k]) for k in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceNorm",
                                                                "faceCenter", "faceArea", "faceXpac", "faceXnac",
                                                                "cellCenter", "cellVolume", "bndRegion", "regionType",
                                                                "regionUVW", "regionDen")])

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.ref_ctx_destroy(self.h)
            self.h = None

    def gradient(self, phi, phib, n_gradient=1, reps=1):
        nc = self.m["nCells"]
        g = np.empty((nc, 3))
        go = np.empty((nc, 3))
        secs = np.empty(reps)
        self._phi = np.ascontiguousarray(phi, np.float64)
        self._phib = np.ascontiguousarray(phib, np.float64)
        rc = self.ref.ref_gradient_phi_gauss(self.h, n_gradient, _p(self._phi), len(self._phi), _p(self._phib),
                                             len(self._phib), _p(g), _p(go), reps, _p(secs))
        return rc, g, go, secs

    def flux_mass(self, f, reps=1):
        out = {k: np.array(f[k], np.float64, copy=True) for k in ("massFlux", "su", "rface", "denB", "teB", "edB", "visB", "tB")}
        cnt = [C.c_int(int(f.get(k, 0))) for k in ("icinl", "icout", "icsym", "icwal")]
        a = {k: np.ascontiguousarray(f[k], np.float64) for k in ("dudx", "dvdx", "dwdx", "dpdx", "den", "u", "v", "w", "p",
                                                                 "ar", "teC", "edC", "visC", "tC")}
        secs = np.empty(reps)
        rc = self.ref.ref_flux_mass_face_loop(
            self.h, _p(a["dudx"]), _p(a["dvdx"]), _p(a["dwdx"]), _p(a["dpdx"]), _p(a["den"]), _p(out["denB"]),
            _p(a["u"]), _p(a["v"]), _p(a["w"]), _p(out["massFlux"]), _p(a["p"]), _p(a["ar"]), _p(out["su"]),
            _p(out["rface"]), float(f["small"]), *[C.byref(c) for c in cnt],
            *[int(bool(f.get(k, False))) for k in ("solveTurbEnergy", "solveTurbDiss", "solveVisc", "solveEnthalpy")],
            _p(a["teC"]), _p(out["teB"]), _p(a["edC"]), _p(out["edB"]), _p(a["visC"]), _p(out["visB"]), _p(a["tC"]),
            _p(out["tB"]), reps, _p(secs))
        out.update(icinl=cnt[0].value, icout=cnt[1].value, icsym=cnt[2].value, icwal=cnt[3].value)
        return rc, out, secs

    # momentum loops, the reference templates called unchanged
    def uvw_geometry(self, rlencos=None, bnd_dist=None):
        self._rl = None if rlencos is None else np.ascontiguousarray(rlencos, np.float64)
        self._bd = None if bnd_dist is None else np.ascontiguousarray(bnd_dist, np.float64)
        self.ref.ref_ctx_set_uvw_geometry(self.h, _p(self._rl), _p(self._bd))
        return self

    def uvw_face_loop1(self, f, reps=1):
        out = {k: _f64(f[k]) for k in UVW_INOUT}
        a = {k: np.ascontiguousarray(f[k], np.float64) for k in ("u", "v", "w", "visC", "visB", "dudx", "dvdx", "dwdx")}
        secs = np.empty(reps)
        rc = self.ref.ref_uvw_face_loop1(
            self.h, float(f["gammaBlend"]), float(f["small"]), _p(a["u"]), _p(a["v"]), _p(a["w"]), _p(out["uB"]),
            _p(out["vB"]), _p(out["wB"]), _p(a["visC"]), _p(a["visB"]), _p(out["massFlux"]), _p(a["dudx"]),
            _p(a["dvdx"]), _p(a["dwdx"]), _p(out["rFace"]), *[_p(out[k]) for k in ("su", "sv", "sw", "au", "av", "aw")],
            reps, _p(secs))
        out["shear"] = self.uvw_state()[0]
        return rc, out, secs

    def uvw_state(self, shear=None, force_tangent=None):
        """Set (when given) and return (shear [nBnd,3], force tangent [nRegions,3])."""
        sh_in = None if shear is None else np.ascontiguousarray(shear, np.float64)
        ft_in = None if force_tangent is None else np.ascontiguousarray(force_tangent, np.float64)
        sh, ft = np.empty((self.m["nBnd"], 3)), np.empty((self.m["nRegions"], 3))
        self.ref.ref_uvw_state(self.h, _p(sh_in), _p(ft_in), _p(sh), _p(ft))
        return sh, ft

    def uvw_region_loop1(self):
        self.ref.ref_uvw_region_loop1(self.h)
        return self.uvw_state()[1]

    def uvw_bnds_loop1(self):
        self.ref.ref_uvw_bnds_loop1(self.h)
        return self.uvw_state()[1]

    # boundary / region loops, the reference templates called unchanged
    def boundary_loops(self, splvl):
        self._splvl = np.ascontiguousarray(splvl, np.float64)
        self.ref.ref_ctx_set_splvl(self.h, _p(self._splvl))
        return self

    def boundary_loop1(self, massflux):
        out = C.c_double(np.nan)
        mf = _f64(massflux)
        assert self.ref.ref_boundary_loop1(self.h, _p(mf), C.byref(out)) == E_SUCCESS
        return out.value

    def boundary_loop2(self, massflux, flow_region):
        out = C.c_double(np.nan)
        mf, fr = _f64(massflux), _f64(flow_region)
        assert self.ref.ref_boundary_loop2(self.h, _p(mf), _p(fr), C.byref(out)) == E_SUCCESS
        return fr, out.value

    def boundary_loop3(self, flowin):
        out = C.c_double(np.nan)
        assert self.ref.ref_boundary_loop3(self.h, float(flowin), C.byref(out)) == E_SUCCESS
        return out.value

    def boundary_loop4(self, massflux, ub, vb, wb, denb, ratearea):
        out = C.c_double(np.nan)
        mf, u, v, w, den = _f64(massflux), _f64(ub), _f64(vb), _f64(wb), _f64(denb)
        assert self.ref.ref_boundary_loop4(self.h, _p(mf), _p(u), _p(v), _p(w), _p(den), float(ratearea),
                                           C.byref(out)) == E_SUCCESS
        return mf, u, v, w, out.value

    def boundary_loop5(self, massflux, su, ub, vb, wb, fact, solve, flow_fact, flowout2):
        out = C.c_double(flowout2)
        mf, s_, u, v, w, ff = _f64(massflux), _f64(su), _f64(ub), _f64(vb), _f64(wb), _f64(flow_fact)
        assert self.ref.ref_boundary_loop5(self.h, _p(mf), _p(s_), _p(u), _p(v), _p(w), float(fact),
                                           *[int(bool(x)) for x in solve], _p(ff), C.byref(out)) == E_SUCCESS
        return mf, s_, u, v, w, out.value

    def boundary_chain(self, massflux, su, ub, vb, wb, denb, flow_region, reps):
        """Per-call seconds of the reference's boundary-loop chain (loops 1, 3,
        4, 2, the region loop, 5) run `reps` times in place (timing only)."""
        a = [_f64(x) for x in (massflux, su, ub, vb, wb, denb, flow_region)]
        ff = np.zeros(self.m["nRegions"])
        secs = np.empty(reps)
        assert self.ref.ref_boundary_chain(self.h, *[_p(x) for x in a], _p(ff), reps, _p(secs)) == E_SUCCESS
        return secs

    def region_loop(self, flow_region, flow_in):
        ff = np.full(self.m["nRegions"], np.nan)
        fr = _f64(flow_region)
        assert self.ref.ref_region_loop(self.h, _p(ff), _p(fr), float(flow_in)) == E_SUCCESS
        return ff


# ---------------------------------------------------------------------------
# seeded synthetic fields (Philox4x32-10 via numpy)
# ---------------------------------------------------------------------------

# momentum face loop: in/out arrays of FluxUVWDolfynFaceLoop1 (UVWKernels.h:45-67)
UVW_INOUT = ("massFlux", "rFace", "su", "sv", "sw", "au", "av", "aw", "uB", "vB", "wB")


def uvw_fields(m, seed):
    """Inputs of the momentum face loop drawn as the reference's benchmark
    draws them (U[1e-6, 1e-2], BenchmarkKernels.cpp:751-815), with signed mass
    fluxes (both upwind branches, the outlet clamp) and seeded velocity
    gradients ~ 1e-2 N(0,1) (the benchmark leaves them unset). rFace starts
    random so untouched entries are checked."""
    nc, nf, nb = m["nCells"], m["nFaces"], m["nBnd"]
    r = np.random.Generator(np.random.Philox(key=seed))
    U = lambda n: r.uniform(1e-6, 1e-2, n)
    f = dict(u=U(nc), v=U(nc), w=U(nc), visC=U(nc), massFlux=U(nf) * r.choice([-1.0, 1.0], nf),
             su=U(nc), sv=U(nc), sw=U(nc), au=U(nc), av=U(nc), aw=U(nc), uB=U(nb), vB=U(nb), wB=U(nb), visB=U(nb),
             dudx=1e-2 * r.standard_normal((nc, 3)), dvdx=1e-2 * r.standard_normal((nc, 3)),
             dwdx=1e-2 * r.standard_normal((nc, 3)), rFace=r.standard_normal(2 * nf), gammaBlend=0.9, small=1e-18)
    return f


def uvw_face_loop1(m, f, rlencos=None, bnd_dist=None):
    """FluxUVWDolfynFaceLoop1 (C restatement). Returns the in/out arrays after
    the call plus the boundary shear [nBnd, 3]."""
    out = {k: _f64(f[k]) for k in UVW_INOUT}
    out["shear"] = np.zeros((m["nBnd"], 3))
    a = {k: np.ascontiguousarray(f[k], np.float64) for k in ("u", "v", "w", "visC", "visB", "dudx", "dvdx", "dwdx")}
    rl = None if rlencos is None else np.ascontiguousarray(rlencos, np.float64)
    bd = None if bnd_dist is None else np.ascontiguousarray(bnd_dist, np.float64)
    rc = load().orc_uvw_face_loop1(C.byref(_cmesh(m)), _p(rl), _p(bd), float(f["gammaBlend"]), float(f["small"]),
                                   _p(a["u"]), _p(a["v"]), _p(a["w"]), _p(out["uB"]), _p(out["vB"]), _p(out["wB"]),
                                   _p(a["visC"]), _p(a["visB"]), _p(out["massFlux"]), _p(a["dudx"]), _p(a["dvdx"]),
                                   _p(a["dwdx"]), _p(out["rFace"]), *[_p(out[k]) for k in ("su", "sv", "sw", "au", "av", "aw")],
                                   _p(out["shear"]))
    assert rc == E_SUCCESS
    return out


class _OrcMeshF(C.Structure):
    _fields_ = [("nCells", C.c_int), ("nFaces", C.c_int), ("nBnd", C.c_int), ("nRegions", C.c_int)] + [
        (n, C.c_void_p) for n in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceNorm", "faceCenter",
                                  "faceArea", "faceXpac", "faceXnac", "cellCenter", "cellVolume", "bndRegion",
                                  "regionType", "regionUVW", "regionDen")]


def _f32(a):
    return None if a is None else np.ascontiguousarray(np.asarray(a).reshape(-1), np.float32)


def _float_mesh(m):
    """Arrays of mesh ``m`` as a CupCfdSoAMesh<int,float,int> holds them
    (float geometry and region values) and an orc_mesh_f over them."""
    keep = {k: np.ascontiguousarray(m[k], np.int32) for k in ("faceCell1", "faceCell2", "faceBnd", "bndRegion",
                                                              "regionType")}
    for k in ("faceLambda", "faceNorm", "faceCenter", "faceArea", "faceXpac", "faceXnac", "cellCenter", "cellVolume",
              "regionUVW", "regionDen"):
        keep[k] = _f32(m[k])
    s = _OrcMeshF(int(m["nCells"]), int(m["nFaces"]), int(m["nBnd"]), int(m["nRegions"]),
                  *[_p(keep[n]) for n, _ in _OrcMeshF._fields_[4:]])
    return s, keep


def _uvw_f32_inputs(f):
    a = {k: _f32(f[k]) for k in ("u", "v", "w", "visC", "visB", "dudx", "dvdx", "dwdx")}
    out = {k: _f32(f[k]).copy() for k in UVW_INOUT}
    return a, out


def uvw_loops_f32(m, f, rlencos=None, bnd_dist=None):
    """The momentum loops of the reference's T = float instantiation (C
    restatement): FluxUVWDolfynFaceLoop1 on float inputs, then the region
    force tangents (zeroed by FluxUVWDolfynRegionLoop1, the wall shears added
    by FluxUVWDolfynBndsLoop1). Returns the in/out arrays (float32), shear
    [nBnd, 3] and the force tangents [nRegions, 3]."""
    s, keep = _float_mesh(m)
    a, out = _uvw_f32_inputs(f)
    out["shear"] = np.zeros((m["nBnd"], 3), np.float32)
    rl, bd = _f32(rlencos), _f32(bnd_dist)
    lib = load()
    lib.orc_uvw_face_loop1_f32.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float] + [C.c_void_p] * 20
    rc = lib.orc_uvw_face_loop1_f32(C.byref(s), _p(rl), _p(bd), float(np.float32(f["gammaBlend"])),
                                    float(np.float32(f["small"])), _p(a["u"]), _p(a["v"]), _p(a["w"]), _p(out["uB"]),
                                    _p(out["vB"]), _p(out["wB"]), _p(a["visC"]), _p(a["visB"]), _p(out["massFlux"]),
                                    _p(a["dudx"]), _p(a["dvdx"]), _p(a["dwdx"]), _p(out["rFace"]),
                                    *[_p(out[k]) for k in ("su", "sv", "sw", "au", "av", "aw")], _p(out["shear"]))
    assert rc == E_SUCCESS
    ft = np.zeros((m["nRegions"], 3), np.float32)
    assert lib.orc_uvw_bnds_loop1_f32(C.byref(s), _p(out["shear"]), _p(ft)) == E_SUCCESS
    out["forceTangent"] = ft
    return out


def ref_uvw_loops_f32(m, f, rlencos=None, bnd_dist=None):
    """The same loops of the reference's own T = float instantiation
    (compiled unchanged), on the same float arrays."""
    ref = load_ref()
    assert ref is not None, "reference build absent"
    _, keep = _float_mesh(m)
    a, out = _uvw_f32_inputs(f)
    nF, nB, nR = int(m["nFaces"]), int(m["nBnd"]), int(m["nRegions"])
    rl = _f32(rlencos) if rlencos is not None else np.zeros(nF, np.float32)
    bd = _f32(bnd_dist) if bnd_dist is not None else np.zeros(nB, np.float32)
    out["shear"] = np.zeros((nB, 3), np.float32)
    out["forceTangent"] = np.full((nR, 3), 7.0, np.float32)
    fn = ref.ref_uvw_loops_f32
    fn.argtypes = [C.c_int] * 4 + [C.c_void_p] * 15 + [C.c_float, C.c_float] + [C.c_void_p] * 21
    geo = [keep[k] for k in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceNorm", "faceCenter", "faceArea",
                             "cellCenter", "cellVolume", "bndRegion", "regionType", "regionUVW", "regionDen")]
    rc = fn(int(m["nCells"]), nF, nB, nR, *[_p(x) for x in geo], _p(rl), _p(bd), float(np.float32(f["gammaBlend"])),
            float(np.float32(f["small"])), _p(a["u"]), _p(a["v"]), _p(a["w"]), _p(out["uB"]), _p(out["vB"]),
            _p(out["wB"]), _p(a["visC"]), _p(a["visB"]), _p(out["massFlux"]), _p(a["dudx"]), _p(a["dvdx"]),
            _p(a["dwdx"]), _p(out["rFace"]), *[_p(out[k]) for k in ("su", "sv", "sw", "au", "av", "aw")],
            _p(out["shear"]), _p(out["forceTangent"]))
    assert rc == E_SUCCESS, rc
    return out


def ref_boundary_chain_f32(m, splvl, d, fact, solve, flowout2):
    """The boundary-loop chain (loops 1, 3, 4, 2, the region loop, 5) of the
    reference's own T = float instantiation (compiled unchanged) on mesh
    ``m``'s float arrays: d holds mf [nFaces], su [nCells], u, v, w, den
    [nBnd], fr [nRegions] (rounded to float). Returns the arrays after
    loop 4 (mf4, u4, v4, w4), loop 2 (fr2), the region loop (ff) and loop 5
    (mf5, su5, u5, v5, w5), and the scalars flowin, ratearea, flowout4,
    flowout2 (loop 2's) and fo2 (loop 5's, continued from ``flowout2``)."""
    ref = load_ref()
    assert ref is not None, "reference build absent"
    _, keep = _float_mesh(m)
    a = {k: _f32(d[k]).copy() for k in ("mf", "su", "u", "v", "w", "den", "fr")}
    nR = int(m["nRegions"])
    ff = np.full(nR, np.nan, np.float32)
    out = np.zeros(5, np.float32)
    sp = _f32(splvl)
    fn = ref.ref_boundary_chain_f32
    fn.argtypes = [C.c_int] * 4 + [C.c_void_p] * 15 + [C.c_float] + [C.c_int] * 3 + [C.c_float, C.c_void_p]
    rc = fn(int(m["nCells"]), int(m["nFaces"]), int(m["nBnd"]), nR, _p(keep["faceCell1"]), _p(keep["faceBnd"]),
            _p(keep["faceNorm"]), _p(keep["faceArea"]), _p(keep["bndRegion"]), _p(keep["regionType"]), _p(sp),
            _p(a["mf"]), _p(a["su"]), _p(a["u"]), _p(a["v"]), _p(a["w"]), _p(a["den"]), _p(a["fr"]), _p(ff),
            float(np.float32(fact)), *[int(bool(x)) for x in solve], float(np.float32(flowout2)), _p(out))
    assert rc == E_SUCCESS, rc
    return dict(mf5=a["mf"], su5=a["su"], u5=a["u"], v5=a["v"], w5=a["w"], fr2=a["fr"], ff=ff,
                flowin=out[0], ratearea=out[1], flowout4=out[2], flowout2=out[3], fo2=out[4])


def uvw_region_loop1(m):
    ft = np.full((m["nRegions"], 3), np.nan)
    assert load().orc_uvw_region_loop1(C.byref(_cmesh(m)), _p(ft)) == E_SUCCESS
    return ft


def uvw_bnds_loop1(m, shear, force_tangent):
    ft = _f64(force_tangent)
    sh = np.ascontiguousarray(shear, np.float64)
    assert load().orc_uvw_bnds_loop1(C.byref(_cmesh(m)), _p(sh), _p(ft)) == E_SUCCESS
    return ft


def fields(m, seed, full=False):
    """phi ~ U[-1,1], u,v,w ~ N(0,1), rho ~ U[0.9,1.1], phiB ~ U[-1,1] from a
    Philox4x32-10 stream keyed by ``seed``. With ``full``, also seeds the
    inputs the plain form holds at zero (velocity/pressure gradients ~ N(0,1),
    p ~ U[-1,1]) and ar ~ U[0.9,1.1]."""
    nc, nf, nb = m["nCells"], m["nFaces"], m["nBnd"]
    r = np.random.Generator(np.random.Philox(key=seed))
    f = dict(phi=r.uniform(-1, 1, nc), u=r.standard_normal(nc), v=r.standard_normal(nc), w=r.standard_normal(nc),
             den=r.uniform(0.9, 1.1, nc), phiB=r.uniform(-1, 1, nb))
    z3 = np.zeros((nc, 3))
    if full:
        f.update(dudx=r.standard_normal((nc, 3)), dvdx=r.standard_normal((nc, 3)), dwdx=r.standard_normal((nc, 3)),
                 dpdx=r.standard_normal((nc, 3)), p=r.uniform(-1, 1, nc), ar=r.uniform(0.9, 1.1, nc))
    else:
        f.update(dudx=z3, dvdx=z3.copy(), dwdx=z3.copy(), dpdx=z3.copy(), p=np.zeros(nc), ar=r.uniform(0.9, 1.1, nc))
    f.update(massFlux=np.zeros(nf), su=np.zeros(nc), rface=np.zeros(2 * nf), denB=np.zeros(nb),
             teC=r.uniform(size=nc), edC=r.uniform(size=nc), visC=r.uniform(size=nc), tC=r.uniform(size=nc),
             teB=np.zeros(nb), edB=np.zeros(nb), visB=np.zeros(nb), tB=np.zeros(nb), small=1e-18,
             solveTurbEnergy=False, solveTurbDiss=False, solveVisc=True, solveEnthalpy=False)
    return f
