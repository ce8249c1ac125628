"""FluxUVWDolfynFaceLoop1, FluxUVWDolfynRegionLoop1 and FluxUVWDolfynBndsLoop1
on the GPU against the oracle, which is itself bit-identical to the
reference's templates (tests/test_oracle_vs_reference.py).

Every output is compared bit for bit: values with their signs (signed zeros
included); NaNs (the zero boundary distances of a MeshSource-built mesh make
the symmetry and wall branches divide by zero) only as NaN, since the NaN
payload an invalid operation produces is the processor's. Meshes:
structured and jittered with permuted numbering, in several cell orders,
random regions with face 0 on an inlet or an outlet (so the reference's
carried face values are defined throughout), and the all-default regions of
a generated mesh (the benchmark's case: interior faces read the carried
values before any face set them, zero here and in the oracle).
"""
import numpy as np
import pytest

import oracle as O
from test_oracle_vs_reference import uvw_case

pytestmark = pytest.mark.gpu


def same(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    return np.array_equal(a[~na].view(np.int64), b[~nb].view(np.int64))


def _mesh(cg, m, order, rl=None, bd=None):
    mesh = cg.Mesh.from_arrays(m, order=order)
    if "regionType" in m:
        assert mesh.set_regions(m["regionType"], m["regionUVW"], m["regionDen"], m["bndRegion"]) == cg.E_SUCCESS
    if rl is not None:
        assert mesh.set_face_rlencos(rl) == cg.E_SUCCESS
    if bd is not None:
        assert mesh.set_boundary_distance(bd) == cg.E_SUCCESS
    return mesh


def _host(cg, mesh, f):
    out = {k: np.array(f[k], np.float64, copy=True) for k in O.UVW_INOUT}
    rc = cg.FluxUVWDolfynFaceLoop1(mesh, f["gammaBlend"], f["small"], f["u"], f["v"], f["w"], out["uB"], out["vB"],
                                   out["wB"], f["visC"], f["visB"], out["massFlux"], f["dudx"], f["dvdx"], f["dwdx"],
                                   out["rFace"], out["su"], out["sv"], out["sw"], out["au"], out["av"], out["aw"])
    assert rc == cg.E_SUCCESS, cg.last_error()
    out["shear"] = mesh.boundary_shear()
    return out


def _check(got, want):
    for k in O.UVW_INOUT + ("shear",):
        assert same(got[k], want[k]), k


@pytest.mark.parametrize("mk,order", [("struct", 0), ("struct", 1), ("jitter", 1), ("jitter", 3)])
@pytest.mark.parametrize("first", ["outlet", "inlet"])
@pytest.mark.parametrize("geom", ["zero", "set"])
def test_uvw_face_loop1_bit_exact(cg, gpu, mk, order, first, geom):
    m, rng = uvw_case(mk, 60 + (mk == "jitter"), first)
    f = O.uvw_fields(m, 62)
    rl = bd = None
    if geom == "set":
        rl = rng.uniform(0.1, 2.0, m["nFaces"])
        bd = rng.uniform(0.01, 0.2, m["nBnd"])
    want = O.uvw_face_loop1(m, f, rl, bd)
    mesh = _mesh(cg, m, order, rl, bd)
    _check(_host(cg, mesh, f), want)
    # the region loops on the shear the face loop left in the mesh
    ft = mesh.region_force_tangent(m["nRegions"], np.full((m["nRegions"], 3), 3.0))
    assert np.all(ft == 3.0)
    assert cg.FluxUVWDolfynRegionLoop1(mesh) == cg.E_SUCCESS
    ft0 = mesh.region_force_tangent(m["nRegions"])
    assert same(ft0, O.uvw_region_loop1(m))
    assert cg.FluxUVWDolfynBndsLoop1(mesh) == cg.E_SUCCESS
    assert same(mesh.region_force_tangent(m["nRegions"]), O.uvw_bnds_loop1(m, want["shear"], ft0))


def same32(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape or a.dtype != np.float32 or b.dtype != np.float32:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(a[~na].view(np.int32), b[~nb].view(np.int32))


@pytest.mark.parametrize("mk,order", [("struct", 1), ("jitter", 3)])
@pytest.mark.parametrize("first", ["outlet", "inlet"])
@pytest.mark.parametrize("geom", ["zero", "set"])
def test_uvw_loops_float_instantiation_bit_exact(cg, gpu, mk, order, first, geom):
    """The momentum loops with T=float arrays on a mesh uploaded from float
    arrays (face loop, region loop, boundary loop in float) against the
    reference's own float build, every output bit for bit."""
    if O.load_ref() is None:
        pytest.skip("reference build absent")
    m, rng = uvw_case(mk, 80 + (mk == "jitter"), first)
    f = O.uvw_fields(m, 83)
    rl = bd = None
    if geom == "set":
        rl = rng.uniform(0.1, 2.0, m["nFaces"]).astype(np.float32)
        bd = rng.uniform(0.01, 0.2, m["nBnd"]).astype(np.float32)
    want = O.ref_uvw_loops_f32(m, f, rl, bd)
    m32 = dict(m)
    for k in ("faceLambda", "faceArea", "faceNorm", "faceCenter", "cellCenter", "cellVolume"):
        m32[k] = np.ascontiguousarray(np.asarray(m[k]), np.float32)
    r32 = dict(m, regionUVW=np.asarray(m["regionUVW"], np.float32).astype(np.float64),
               regionDen=np.asarray(m["regionDen"], np.float32).astype(np.float64))
    mesh = cg.Mesh.from_arrays(m32, order=order)
    assert mesh.set_regions(r32["regionType"], r32["regionUVW"], r32["regionDen"], r32["bndRegion"]) == cg.E_SUCCESS
    if rl is not None:
        assert mesh.set_face_rlencos(rl.astype(np.float64)) == cg.E_SUCCESS
        assert mesh.set_boundary_distance(bd.astype(np.float64)) == cg.E_SUCCESS
    g = {k: np.ascontiguousarray(f[k], np.float32) for k in ("u", "v", "w", "visC", "visB", "dudx", "dvdx", "dwdx")}
    out = {k: np.array(f[k], np.float32, copy=True) for k in O.UVW_INOUT}
    rc = cg.FluxUVWDolfynFaceLoop1(mesh, np.float32(f["gammaBlend"]), np.float32(f["small"]), g["u"], g["v"], g["w"],
                                   out["uB"], out["vB"], out["wB"], g["visC"], g["visB"], out["massFlux"], g["dudx"],
                                   g["dvdx"], g["dwdx"], out["rFace"], out["su"], out["sv"], out["sw"], out["au"],
                                   out["av"], out["aw"])
    assert rc == cg.E_SUCCESS, cg.last_error()
    for k in O.UVW_INOUT:
        assert same32(out[k], want[k]), k
    assert same32(mesh.boundary_shear().astype(np.float32), want["shear"])
    mesh.region_force_tangent(m["nRegions"], np.full((m["nRegions"], 3), 7.0))
    assert cg.FluxUVWDolfynRegionLoop1(mesh) == cg.E_SUCCESS
    assert cg.FluxUVWDolfynBndsLoop1(mesh) == cg.E_SUCCESS
    assert same32(mesh.region_force_tangent(m["nRegions"]).astype(np.float32), want["forceTangent"])


@pytest.mark.parametrize("order", [0, 1, 3])
def test_uvw_default_regions(cg, gpu, order):
    """The generated mesh with its single default region (what the
    reference's benchmark runs): only interior faces contribute, their
    carried uFace is zero before any inlet/outlet face."""
    m = O.structgen(13, 9, 7)
    f = O.uvw_fields(m, 63)
    want = O.uvw_face_loop1(m, f)
    mesh = _mesh(cg, m, order)
    _check(_host(cg, mesh, f), want)


def test_uvw_first_faces_unset(cg, gpu):
    """Face 0 on a symmetry face and interior faces before the first inlet:
    the GPU follows the oracle's zero start for the carried values."""
    base = O.jitter(9, 8, 7, 0.25, seed=5, permute=True)
    m, _, rng = __import__("test_oracle_vs_reference")._with_regions(base, 77)
    m["bndRegion"][m["faceBnd"][0]] = 3
    f = O.uvw_fields(m, 64)
    rl, bd = rng.uniform(0.1, 2.0, m["nFaces"]), rng.uniform(0.01, 0.2, m["nBnd"])
    want = O.uvw_face_loop1(m, f, rl, bd)
    _check(_host(cg, _mesh(cg, m, 1, rl, bd), f), want)


def test_uvw_regions_changed(cg, gpu):
    """Changing the regions after a call rebuilds the carried-value sources."""
    m, rng = uvw_case("struct", 65, "outlet")
    f = O.uvw_fields(m, 66)
    mesh = _mesh(cg, m, 1)
    _check(_host(cg, mesh, f), O.uvw_face_loop1(m, f))
    m2 = dict(m)
    m2["bndRegion"] = rng.integers(0, m["nRegions"], m["nBnd"]).astype(np.int32)
    m2["bndRegion"][m["faceBnd"][0]] = 1
    assert mesh.set_regions(m2["regionType"], m2["regionUVW"], m2["regionDen"], m2["bndRegion"]) == cg.E_SUCCESS
    mesh.boundary_shear(np.zeros((m["nBnd"], 3)))
    _check(_host(cg, mesh, f), O.uvw_face_loop1(m2, f))


@pytest.mark.parametrize("order", [1, 3])
def test_uvw_device_equals_host(cg, gpu, order):
    import torch
    dev = torch.device("cuda:0")
    m, rng = uvw_case("jitter", 67, "outlet")
    f = O.uvw_fields(m, 68)
    rl, bd = rng.uniform(0.1, 2.0, m["nFaces"]), rng.uniform(0.01, 0.2, m["nBnd"])
    mesh = _mesh(cg, m, order, rl, bd)
    host = _host(cg, mesh, f)
    mesh.boundary_shear(np.zeros((m["nBnd"], 3)))
    c2o, f2o = mesh.numbering()

    def T(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    cells = {k: T(f[k][c2o]) for k in ("u", "v", "w", "visC", "su", "sv", "sw", "au", "av", "aw")}
    grads = T(np.concatenate([f[k][c2o].T for k in ("dudx", "dvdx", "dwdx")]))
    assert grads.shape == (9, m["nCells"])
    bnd = {k: T(f[k]) for k in ("uB", "vB", "wB", "visB")}
    mf = T(f["massFlux"][f2o])
    rf = T(f["rFace"].reshape(-1, 2)[f2o].reshape(-1))
    s = torch.cuda.current_stream()
    cg.dev_uvw_face_loop1(mesh, f["gammaBlend"], f["small"], cells["u"], cells["v"], cells["w"], bnd["uB"], bnd["vB"],
                          bnd["wB"], cells["visC"], bnd["visB"], mf, grads, rf, cells["su"], cells["sv"], cells["sw"],
                          cells["au"], cells["av"], cells["aw"], stream=s)
    torch.cuda.synchronize()

    def to_ref(t, n2o, width=1):
        a = t.cpu().numpy().reshape(len(n2o), width)
        out = np.empty_like(a)
        out[n2o] = a
        return out.reshape(-1) if width > 1 else out[:, 0]

    for k in ("su", "sv", "sw", "au", "av", "aw"):
        assert same(to_ref(cells[k], c2o), host[k]), k
    assert same(to_ref(mf, f2o), host["massFlux"])
    assert same(to_ref(rf, f2o, 2), host["rFace"])
    for k in ("uB", "vB", "wB"):
        assert same(bnd[k].cpu().numpy(), host[k]), k
    assert same(mesh.boundary_shear(), host["shear"])


def test_uvw_errors(cg, gpu):
    m, _ = uvw_case("struct", 69, "outlet")
    f = O.uvw_fields(m, 70)
    mesh = _mesh(cg, m, 1)
    o = {k: np.array(f[k], np.float64, copy=True) for k in O.UVW_INOUT}
    args = (f["u"], f["v"], f["w"], o["uB"], o["vB"], o["wB"], f["visC"], f["visB"], o["massFlux"], f["dudx"], f["dvdx"],
            f["dwdx"], o["rFace"][:-1].copy(), o["su"], o["sv"], o["sw"], o["au"], o["av"], o["aw"])
    assert cg.FluxUVWDolfynFaceLoop1(mesh, 0.9, 1e-18, *args) == cg.E_INVALID_INDEX
    assert cg.last_error().startswith("FluxUVWDolfynFaceLoop1: array shorter")
    assert np.array_equal(o["su"], f["su"])   # nothing written
    assert mesh.set_face_rlencos(np.zeros(m["nFaces"] - 1)) == cg.E_ARRAY_SIZE_MISMATCH
    assert mesh.set_boundary_distance(np.zeros(m["nBnd"] + 1)) == cg.E_ARRAY_SIZE_MISMATCH
    with pytest.raises(cg.CupcfdError):
        mesh.region_force_tangent(m["nRegions"] + 1)


def test_uvw_large_jittered_permuted(cg, gpu):
    """A 128^3 jittered mesh with permuted numbering (2,097,152 cells,
    6,340,608 faces), six random regions, set rlencos and boundary distances,
    in reverse Cuthill-McKee order: every output bit for bit against the
    oracle, and the region / boundary loops after it."""
    from test_oracle_vs_reference import _with_regions
    base = O.jitter(128, 128, 128, 0.25, seed=9, permute=True)
    m, _, rng = _with_regions(base, 90)
    f = O.uvw_fields(m, 91)
    rl, bd = rng.uniform(0.1, 2.0, m["nFaces"]), rng.uniform(0.01, 0.2, m["nBnd"])
    want = O.uvw_face_loop1(m, f, rl, bd)
    mesh = _mesh(cg, m, cg.ORDER_RCM, rl, bd)
    _check(_host(cg, mesh, f), want)
    assert cg.FluxUVWDolfynRegionLoop1(mesh) == cg.E_SUCCESS
    ft0 = mesh.region_force_tangent(m["nRegions"])
    assert same(ft0, O.uvw_region_loop1(m))
    assert cg.FluxUVWDolfynBndsLoop1(mesh) == cg.E_SUCCESS
    assert same(mesh.region_force_tangent(m["nRegions"]), O.uvw_bnds_loop1(m, want["shear"], ft0))
