"""Parity of the CUDA library (through the C ABI) with the oracle.

FP64 path: bit-identical to the oracle, which is itself bit-identical to the
reference's own CPU kernels (tests/test_oracle_vs_reference.py). The stated
contract is <= 1e-12 relative; the tests assert equality of every element.

FP32-compensated path: FP32 fields and geometry, compensated (TwoSum, after
Dot2) accumulation, FP64 volumes. Measured against the FP64 oracle fed the
same FP32-rounded inputs.
Tolerances:
  normwise   max|d| / max|ref|                      <= 1e-6
  rms        ||d||_2 / ||ref||_2                    <= 1e-6
  elementwise max |d| / max(|ref|, 1e-2 * rms(ref)) <= 1e-5 forward, 5e-5 adjoint
Each face term carries one FP32 rounding (about 6e-8 of the term); a cell
sum of six terms that cancels down to 1e-2 of the typical magnitude turns
that into ~1e-5 relative, and the adjoint sums (two interpolations per term)
reach a few 1e-5. The sums themselves are compensated and add nothing.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

ORDERS = [0, 1, 2, 3]  # native, morton, owner, rcm


def vec4(n):
    """(n,4) host array emulating std::vector<EuclideanVector<double,3>>: a
    pad slot where the vptr sits, then the 3 components (32-byte stride)."""
    a = np.full((n, 4), np.nan)
    return a


def as_f32(x):
    return np.asarray(x, np.float32).astype(np.float64)


def errs(got, ref):
    got, ref = np.asarray(got, np.float64).ravel(), np.asarray(ref, np.float64).ravel()
    d = np.abs(got - ref)
    mref = np.abs(ref).max()
    rms = np.sqrt(np.mean(ref ** 2))
    return dict(norm=d.max() / mref if mref else d.max(),
                rms=np.linalg.norm(got - ref) / np.linalg.norm(ref) if np.any(ref) else 0.0,
                elem=(d / np.maximum(np.abs(ref), 1e-2 * rms)).max() if rms else d.max())


def assert_f32c(got, ref, what, elem=1e-5):
    e = errs(got, ref)
    assert e["norm"] <= 1e-6 and e["rms"] <= 1e-6 and e["elem"] <= elem, (what, e)


def assert_incidences_match(mesh, ref):
    """The renumbered incidence lists the kernels read, mapped back through
    the mesh's numbering, equal the reference's cell->face CSR row by row and
    in order, with each entry's role and other cell (or boundary id) taken
    from the reference's faceCell1 / faceCell2 / faceBnd."""
    xadj, face, other = mesh.incidences()
    c2o, f2o = mesh.numbering()
    rx, ra = O.cell_face_csr(ref)
    lens = np.diff(xadj)
    assert np.array_equal(lens, rx[c2o + 1] - rx[c2o])
    idx = np.repeat(rx[c2o] - xadj[:-1], lens) + np.arange(len(face))
    F = f2o[face >> 1]
    assert np.array_equal(F, ra[idx])
    cell = np.repeat(c2o, lens)
    role = face & 1
    c1, c2, bnd = ref["faceCell1"][F], ref["faceCell2"][F], ref["faceBnd"][F]
    assert np.array_equal(np.where(role == 0, c1, c2), cell)
    inner = other >= 0
    assert np.array_equal(inner, c2 >= 0)
    assert np.array_equal(c2o[other[inner]], np.where(role == 0, c2, c1)[inner])
    assert np.array_equal(-1 - other[~inner], bnd[~inner])


# ---------------------------------------------------------------------------
# mesh construction
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 3, 4), (16, 16, 16), (13, 7, 5)])
@pytest.mark.parametrize("order", ORDERS)
def test_structgen_on_gpu_equals_oracle(cg, gpu, dims, order):
    bounds = (-1.0, 1.0, -1.0, 2.0, 0.0, 2.0)
    mesh = cg.Mesh.structgen(*dims, bounds=bounds, order=order)
    ref = O.structgen(*dims, bounds=bounds)
    g = mesh.geometry()
    for k in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceArea", "faceNorm", "faceCenter", "cellCenter",
              "cellVolume"):
        assert np.array_equal(g[k], ref[k]), k
    xadj, adj = mesh.cell_face_csr()
    rx, ra = O.cell_face_csr(ref)
    assert np.array_equal(xadj, rx) and np.array_equal(adj, ra)
    assert_incidences_match(mesh, ref)
    assert mesh.nInteriorFaces == int(np.count_nonzero(ref["faceCell2"] >= 0))
    c, f = mesh.numbering()
    assert np.array_equal(np.sort(c), np.arange(mesh.nCells)) and np.array_equal(np.sort(f), np.arange(mesh.nFaces))
    if order == 0:
        assert np.array_equal(c, np.arange(mesh.nCells)) and np.array_equal(f, np.arange(mesh.nFaces))


@pytest.mark.parametrize("order", ORDERS)
def test_uploaded_mesh_roundtrip(cg, gpu, order):
    ref = O.jitter(7, 6, 5, 0.25, seed=3, permute=True)
    m = dict(ref)
    for k in ("faceNorm", "faceCenter", "cellCenter"):     # EuclideanVector layout: 32-byte stride
        a = vec4(len(ref[k]))
        a[:, 1:] = ref[k]
        m[k] = a
    mesh = cg.Mesh.from_arrays(m, order=order)
    g = mesh.geometry()
    for k in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceArea", "faceNorm", "faceCenter", "cellCenter",
              "cellVolume"):
        assert np.array_equal(g[k], ref[k]), k
    xadj, adj = mesh.cell_face_csr()
    rx, ra = O.cell_face_csr(ref)
    assert np.array_equal(xadj, rx) and np.array_equal(adj, ra)
    assert_incidences_match(mesh, ref)


@pytest.mark.parametrize("permute", [False, True])
def test_jittered_on_gpu_equals_oracle(cg, gpu, permute):
    ref = O.jitter(9, 8, 7, 0.25, seed=11, permute=permute)
    mesh = cg.Mesh.jittered(9, 8, 7, 0.25, seed=11, permute=permute)
    g = mesh.geometry()
    for k in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceArea", "faceNorm", "faceCenter", "cellCenter",
              "cellVolume"):
        assert np.array_equal(g[k], ref[k]), k


# ---------------------------------------------------------------------------
# GradientPhiGaussDolfyn, FP64: bit-identical
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 3, 4), (16, 16, 16), (13, 7, 5)])
@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("ngrad", [0, 1, 2, 3])
def test_gradient_f64_bit_exact(cg, gpu, dims, order, ngrad):
    ref = O.structgen(*dims)
    mesh = cg.Mesh.structgen(*dims, order=order)
    f = O.fields(ref, 100 + ngrad)
    rc, g_ref, go_ref = O.gradient(ref, f["phi"], f["phiB"], ngrad)
    n = ref["nCells"]
    g, go = vec4(n), vec4(n)
    g[:, 1:] = 7.0                      # untouched when nGradient = 0
    rc2 = cg.GradientPhiGaussDolfyn(mesh, ngrad, f["phi"], f["phiB"], g, go)
    assert rc == rc2 == cg.E_SUCCESS
    assert np.all(np.isnan(g[:, 0])) and np.all(np.isnan(go[:, 0]))    # the vptr slot is never written
    if ngrad == 0:
        assert np.all(g[:, 1:] == 7.0)
    else:
        assert np.array_equal(g[:, 1:], g_ref)
    assert np.array_equal(go[:, 1:], go_ref)


@pytest.mark.parametrize("ngrad", [1, 2])
def test_gradient_f64_permuted_jittered_bit_exact(cg, gpu, ngrad):
    ref = O.jitter(12, 10, 9, 0.25, seed=5, permute=True)
    f = O.fields(ref, 77)
    rc, g_ref, go_ref = O.gradient(ref, f["phi"], f["phiB"], ngrad)
    for mesh in (cg.Mesh.from_arrays(ref), cg.Mesh.jittered(12, 10, 9, 0.25, seed=5, permute=True)):
        g, go = np.empty((ref["nCells"], 3)), np.empty((ref["nCells"], 3))
        assert cg.GradientPhiGaussDolfyn(mesh, ngrad, f["phi"], f["phiB"], g, go) == cg.E_SUCCESS
        assert np.array_equal(g, g_ref) and np.array_equal(go, go_ref)


def test_gradient_f64_128cubed_bit_exact(cg, gpu):
    """The plain-FP64 configuration: 128^3 structured mesh."""
    ref = O.structgen(128, 128, 128)
    mesh = cg.Mesh.structgen(128, 128, 128)
    f = O.fields(ref, 20261204)
    rc, g_ref, _ = O.gradient(ref, f["phi"], f["phiB"], 1)
    g, go = np.empty((ref["nCells"], 3)), np.empty((ref["nCells"], 3))
    assert cg.GradientPhiGaussDolfyn(mesh, 1, f["phi"], f["phiB"], g, go) == cg.E_SUCCESS
    assert np.array_equal(g, g_ref)
    mf = O.mass_plain(ref, f["den"], f["u"], f["v"], f["w"])
    out = cg.forward_adjoint(mesh, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"],
                             np.zeros(ref["nFaces"]))
    assert np.array_equal(out["massFlux"], mf)
    assert np.array_equal(out["grad"], g_ref)


def test_gradient_signed_mode(cg, gpu):
    """SIGN_SIGNED: neighbour subtracts (textbook Gauss-Green); a linear field
    then has its exact gradient in every interior cell."""
    dims = (8, 8, 8)
    ref = O.structgen(*dims)
    mesh = cg.Mesh.structgen(*dims)
    x = ref["cellCenter"]
    a = np.array([0.3, -1.2, 2.5])
    phi = x @ a + 0.7
    # boundary value: the linear field at the boundary face centre
    bfaces = np.nonzero(ref["faceBnd"] >= 0)[0]
    phib = np.empty(ref["nBnd"])
    phib[ref["faceBnd"][bfaces]] = ref["faceCenter"][bfaces] @ a + 0.7
    g, go = np.empty((ref["nCells"], 3)), np.empty((ref["nCells"], 3))
    assert cg.GradientPhiGaussDolfyn(mesh, 1, phi, phib, g, go, sign_mode=cg.SIGN_SIGNED) == cg.E_SUCCESS
    assert np.allclose(g, a[None, :], rtol=0, atol=1e-12)


# ---------------------------------------------------------------------------
# FluxMassDolfynFaceLoop, full semantics, FP64: bit-identical
# ---------------------------------------------------------------------------
def _mass_case(cg, mesh, ref, f):
    cnt = np.array([3, 0, 1, 0], np.int32)
    out = {k: np.array(f[k], np.float64, copy=True) for k in ("massFlux", "su", "rface", "denB", "teB", "edB", "visB", "tB")}
    vv = {}
    for k in ("dudx", "dvdx", "dwdx", "dpdx"):
        a = vec4(ref["nCells"])
        a[:, 1:] = f[k]
        vv[k] = a
    rc = cg.FluxMassDolfynFaceLoop(mesh, vv["dudx"], vv["dvdx"], vv["dwdx"], vv["dpdx"], f["den"], out["denB"], f["u"],
                                   f["v"], f["w"], out["massFlux"], f["p"], f["ar"], out["su"], out["rface"], f["small"],
                                   cnt, f["solveTurbEnergy"], f["solveTurbDiss"], f["solveVisc"], f["solveEnthalpy"],
                                   f["teC"], out["teB"], f["edC"], out["edB"], f["visC"], out["visB"], f["tC"], out["tB"])
    out.update(icinl=int(cnt[0]), icout=int(cnt[1]), icsym=int(cnt[2]), icwal=int(cnt[3]))
    return rc, out


@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("regions", [False, True])
@pytest.mark.parametrize("jit", [False, True])
def test_mass_full_f64_bit_exact(cg, gpu, order, regions, jit):
    ref = O.jitter(9, 7, 8, 0.25, seed=2, permute=True) if jit else O.structgen(9, 7, 8)
    mesh = cg.Mesh.from_arrays(ref, order=order)
    if regions:
        ref = dict(ref)
        rng = np.random.default_rng(8)
        ref["nRegions"] = 5
        ref["regionType"] = np.array([0, 1, 2, 3, 4], np.int32)
        ref["regionUVW"] = rng.standard_normal((5, 3))
        ref["regionDen"] = rng.uniform(0.5, 1.5, 5)
        ref["bndRegion"] = rng.integers(0, 5, ref["nBnd"]).astype(np.int32)
        assert mesh.set_regions(ref["regionType"], ref["regionUVW"], ref["regionDen"], ref["bndRegion"]) == cg.E_SUCCESS
    f = O.fields(ref, 31, full=True)
    f["massFlux"] = np.random.default_rng(1).standard_normal(ref["nFaces"])   # boundary entries must survive
    f["solveTurbEnergy"] = f["solveEnthalpy"] = True
    f["icinl"], f["icsym"] = 3, 1
    rc, o_ref = O.flux_mass_face_loop(ref, f)
    rc2, o = _mass_case(cg, mesh, ref, f)
    assert rc == rc2 == cg.E_SUCCESS
    for k in ("massFlux", "su", "rface", "denB", "teB", "edB", "visB", "tB"):
        assert np.array_equal(o[k], o_ref[k]), k
    for k in ("icinl", "icout", "icsym", "icwal"):
        assert o[k] == o_ref[k], k


@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("jit", [False, True])
@pytest.mark.parametrize("xpac", [False, True])
def test_mass_float_instantiation_bit_exact(cg, gpu, order, jit, xpac):
    """FluxMassDolfynFaceLoop with T=float arrays on a mesh uploaded from float
    arrays against the reference's own T=float instantiation (compiled
    unchanged): every output bit for bit, with all four region types, the
    outlet backflow copies and (xpac) nonzero xpac / xnac."""
    if O.load_ref() is None:
        pytest.skip("reference build absent")
    ref = O.jitter(9, 7, 8, 0.25, seed=2, permute=True) if jit else O.structgen(9, 7, 8)
    ref = dict(ref)
    rng = np.random.default_rng(81)
    ref["nRegions"] = 5
    ref["regionType"] = np.array([0, 1, 2, 3, 4], np.int32)
    ref["regionUVW"] = rng.standard_normal((5, 3))
    ref["regionDen"] = rng.uniform(0.5, 1.5, 5)
    ref["bndRegion"] = rng.integers(0, 5, ref["nBnd"]).astype(np.int32)
    if xpac:
        ref["faceXpac"] = np.asarray(ref["faceCenter"]) + 0.01 * rng.standard_normal((ref["nFaces"], 3))
        ref["faceXnac"] = np.asarray(ref["faceCenter"]) + 0.01 * rng.standard_normal((ref["nFaces"], 3))
    m32 = dict(ref)
    for k in ("faceLambda", "faceArea", "faceNorm", "faceCenter", "faceXpac", "faceXnac", "cellCenter", "cellVolume",
              "regionUVW", "regionDen"):
        m32[k] = np.ascontiguousarray(np.asarray(ref[k]), np.float32)
    mesh = cg.Mesh.from_arrays(m32, order=order)
    assert mesh.set_regions(ref["regionType"], m32["regionUVW"].astype(np.float64), m32["regionDen"].astype(np.float64),
                            ref["bndRegion"]) == cg.E_SUCCESS
    f = O.fields(ref, 82, full=True)
    f["massFlux"] = rng.standard_normal(ref["nFaces"])   # boundary entries must survive
    f["solveTurbEnergy"] = f["solveTurbDiss"] = f["solveEnthalpy"] = True
    f32 = {k: (np.ascontiguousarray(v, np.float32) if isinstance(v, np.ndarray) else v) for k, v in f.items()}
    rc, want = O.ref_flux_mass_f32(m32, f32)
    out = {k: np.array(f32[k], np.float32, copy=True) for k in ("massFlux", "su", "rface", "denB", "teB", "edB", "visB", "tB")}
    cnt = np.zeros(4, np.int32)
    rc2 = cg.FluxMassDolfynFaceLoop(mesh, f32["dudx"], f32["dvdx"], f32["dwdx"], f32["dpdx"], f32["den"], out["denB"],
                                    f32["u"], f32["v"], f32["w"], out["massFlux"], f32["p"], f32["ar"], out["su"],
                                    out["rface"], np.float32(f["small"]), cnt, True, True, True, True, f32["teC"],
                                    out["teB"], f32["edC"], out["edB"], f32["visC"], out["visB"], f32["tC"], out["tB"])
    assert rc == rc2 == cg.E_SUCCESS, cg.last_error()
    for k in ("massFlux", "su", "rface", "denB", "teB", "edB", "visB", "tB"):
        assert np.array_equal(out[k].view(np.int32), want[k].view(np.int32)), k
    assert list(cnt) == [want["icinl"], want["icout"], want["icsym"], want["icwal"]]
    assert want["icinl"] > 0 and want["icout"] > 0 and want["icsym"] > 0 and want["icwal"] > 0

# ---------------------------------------------------------------------------
# FP32-compensated path: error bounds against the FP64 oracle
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("mk", ["struct32", "struct13x7x5", "jitter"])
def test_f32c_forward_error_bounds(cg, gpu, mk):
    if mk == "struct32":
        ref, mesh = O.structgen(32, 32, 32), cg.Mesh.structgen(32, 32, 32)
    elif mk == "struct13x7x5":
        ref, mesh = O.structgen(13, 7, 5), cg.Mesh.structgen(13, 7, 5)
    else:
        ref = O.jitter(20, 18, 16, 0.25, seed=9, permute=True)
        mesh = cg.Mesh.jittered(20, 18, 16, 0.25, seed=9, permute=True)
    f = {k: as_f32(v) if isinstance(v, np.ndarray) and v.dtype == np.float64 else v for k, v in O.fields(ref, 42).items()}
    # the oracle sees FP32-rounded geometry too
    r32 = dict(ref)
    for k in ("faceNorm", "faceLambda"):
        r32[k] = as_f32(ref[k])
    rc, g_ref, _ = O.gradient(r32, f["phi"], f["phiB"], 1)
    mf_ref = O.mass_plain(r32, f["den"], f["u"], f["v"], f["w"])
    out = cg.forward_adjoint(mesh, cg.PREC_F32C, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"],
                             np.zeros(ref["nFaces"]))
    assert_f32c(out["grad"], g_ref, "gradient")
    inner = ref["faceCell2"] >= 0
    assert_f32c(out["massFlux"][inner], mf_ref[inner], "mass flux")
    g2, go2 = np.empty_like(g_ref), np.empty_like(g_ref)
    assert cg.GradientPhiGaussDolfyn(mesh, 1, f["phi"], f["phiB"], g2, go2, precision=cg.PREC_F32C) == cg.E_SUCCESS
    assert_f32c(g2, g_ref, "gradient (reference-facing call)")


# ---------------------------------------------------------------------------
# adjoints
# ---------------------------------------------------------------------------
def _loss_oracle(ref, f, gface):
    rc, g, _ = O.gradient(ref, f["phi"], f["phiB"], 1)
    mf = O.mass_plain(ref, f["den"], f["u"], f["v"], f["w"])
    inner = ref["faceCell2"] >= 0
    return float(np.sum(ref["cellVolume"][:, None] * g * g) + np.sum(gface[inner] * mf[inner])), g, mf


def _adjoint_oracle(ref, f, gface):
    rc, g, _ = O.gradient(ref, f["phi"], f["phiB"], 1)
    pb, pbb = O.gradient_adjoint(ref, 2.0 * ref["cellVolume"][:, None] * g)
    db, ub, vb, wb = O.mass_plain_adjoint(ref, f["den"], f["u"], f["v"], f["w"], gface)
    return dict(phiBar=pb, phiBBar=pbb, denBar=db, uBar=ub, vBar=vb, wBar=wb)


@pytest.mark.parametrize("mk", ["struct", "jitter"])
def test_adjoint_f64_matches_oracle(cg, gpu, mk):
    if mk == "struct":
        ref, mesh = O.structgen(12, 11, 10), cg.Mesh.structgen(12, 11, 10)
    else:
        ref = O.jitter(12, 11, 10, 0.25, seed=6, permute=True)
        mesh = cg.Mesh.jittered(12, 11, 10, 0.25, seed=6, permute=True)
    f = O.fields(ref, 7)
    gface = np.random.Generator(np.random.Philox(key=8)).standard_normal(ref["nFaces"])
    out = cg.forward_adjoint(mesh, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    A = _adjoint_oracle(ref, f, gface)
    L, _, _ = _loss_oracle(ref, f, gface)
    for k, v in A.items():
        e = errs(out[k], v)
        assert e["norm"] <= 1e-13 and e["rms"] <= 1e-13, (k, e)
    assert abs(out["loss"][0] - L) <= 1e-12 * abs(L)


def test_adjoint_f64_central_differences(cg, gpu):
    """Directional derivatives of L along 64 seeded random directions:
    central differences (eps = 1e-6, FP64, evaluated by the oracle's forward)
    agree with <grad L, d> from the GPU adjoint to 1e-6 relative."""
    ref = O.jitter(8, 7, 6, 0.25, seed=12, permute=True)
    mesh = cg.Mesh.from_arrays(ref)
    f = O.fields(ref, 70)
    gface = np.random.Generator(np.random.Philox(key=71)).standard_normal(ref["nFaces"])
    out = cg.forward_adjoint(mesh, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    rng = np.random.Generator(np.random.Philox(key=72))
    keys = ("phi", "phiB", "den", "u", "v", "w")
    bars = dict(phi="phiBar", phiB="phiBBar", den="denBar", u="uBar", v="vBar", w="wBar")
    eps = 1e-6
    worst = 0.0
    for _ in range(64):
        d = {k: rng.standard_normal(len(f[k])) for k in keys}
        fp = dict(f, **{k: f[k] + eps * d[k] for k in keys})
        fm = dict(f, **{k: f[k] - eps * d[k] for k in keys})
        fd = (_loss_oracle(ref, fp, gface)[0] - _loss_oracle(ref, fm, gface)[0]) / (2 * eps)
        ad = sum(float(np.dot(out[bars[k]], d[k])) for k in keys)
        worst = max(worst, abs(fd - ad) / max(abs(ad), 1e-30))
    assert worst <= 1e-6, worst


def test_adjoint_f32c_error_bounds(cg, gpu):
    ref = O.structgen(24, 20, 16)
    mesh = cg.Mesh.structgen(24, 20, 16)
    f = {k: as_f32(v) if isinstance(v, np.ndarray) and v.dtype == np.float64 else v for k, v in O.fields(ref, 3).items()}
    gface = as_f32(np.random.Generator(np.random.Philox(key=4)).standard_normal(ref["nFaces"]))
    out = cg.forward_adjoint(mesh, cg.PREC_F32C, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    r32 = dict(ref)
    for k in ("faceNorm", "faceLambda"):
        r32[k] = as_f32(ref[k])
    # the FP32 path's gradient feeds its adjoint; the FP64 reference adjoint
    # is evaluated at the FP64 gradient of the same inputs
    A = _adjoint_oracle(r32, f, gface)
    for k, v in A.items():
        assert_f32c(out[k], v, k, elem=5e-5)


def test_torch_autograd_binding(cg, gpu):
    """The autograd binding (used only for checking) reproduces the adjoint
    through torch.autograd on device tensors."""
    import torch
    from cupcfd_b200 import autograd as AG
    ref = O.structgen(6, 5, 4)
    mesh = cg.Mesh.structgen(6, 5, 4, order=cg.ORDER_MORTON)
    f = O.fields(ref, 9)
    dev = torch.device("cuda:0")
    nC = ref["nCells"]
    phi_ref = torch.tensor(f["phi"], device=dev)
    st_ref = torch.tensor(np.stack([f["den"], f["u"], f["v"], f["w"]]), device=dev)
    phi = torch.empty(nC, dtype=torch.float64, device=dev)
    st = torch.empty(4, nC, dtype=torch.float64, device=dev)
    cg.permute_cells(mesh, True, phi_ref, phi)
    cg.permute_cells(mesh, True, st_ref, st, ncomp=4)
    phiB = torch.tensor(f["phiB"], device=dev)
    phi.requires_grad_(True)
    st.requires_grad_(True)
    phiB.requires_grad_(True)
    assert torch.autograd.gradcheck(lambda a, b: AG.gradient(mesh, a, b), (phi, phiB), eps=1e-6, atol=1e-8)
    assert torch.autograd.gradcheck(lambda s: AG.mass_flux(mesh, s), (st,), eps=1e-6, atol=1e-8)


# ---------------------------------------------------------------------------
# forward + adjoint: the one call against the separate forward and adjoint
# ---------------------------------------------------------------------------
def _dev_fields(mesh, prec, seed):
    import torch
    dev = torch.device("cuda:0")
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    dt = torch.float64 if prec == 0 else torch.float32
    nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
    phi = (torch.rand(nC, generator=g, device=dev, dtype=torch.float64) * 2 - 1).to(dt)
    phiB = (torch.rand(nB, generator=g, device=dev, dtype=torch.float64) * 2 - 1).to(dt)
    st = torch.randn(4, nC, generator=g, device=dev, dtype=torch.float64).to(dt)
    if prec == 1:
        st = st.t().contiguous()                 # float4 per cell
    gface = torch.randn(nF, generator=g, device=dev, dtype=torch.float64).to(dt)
    return phi, phiB, st, gface


def _run_fa(cg, mesh, prec, fields, separate):
    """dev_forward_adjoint (separate False) or dev_forward + dev_adjoint."""
    import torch
    phi, phiB, st, gface = fields
    nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
    dt = phi.dtype
    out = dict(grad=torch.full((3, nC), float("nan"), dtype=dt, device=phi.device),
               mflux=torch.zeros(nF, dtype=dt, device=phi.device),
               pb=torch.full((nC,), float("nan"), dtype=dt, device=phi.device),
               pbb=torch.full((nB,), float("nan"), dtype=dt, device=phi.device),
               sb=torch.full_like(st, float("nan")),
               loss=torch.zeros(1, dtype=torch.float64, device=phi.device))
    s = torch.cuda.current_stream()
    if separate:
        cg.dev_forward(mesh, prec, phi, phiB, st, out["grad"], out["mflux"], gface=gface, loss=out["loss"], stream=s)
        cg.dev_adjoint(mesh, prec, out["grad"], st, gface, out["pb"], out["pbb"], out["sb"], stream=s)
    else:
        cg.dev_forward_adjoint(mesh, prec, phi, phiB, st, gface, out["grad"], out["mflux"], out["pb"], out["pbb"],
                               out["sb"], out["loss"], stream=s)
    assert mesh.check_status(torch.cuda.current_stream()) == cg.E_SUCCESS
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("order", [0, 1, 2, 3])
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("mk", ["struct", "jitter"])
def test_forward_adjoint_equals_separate_calls(cg, gpu, order, prec, mk):
    import torch
    mesh = (cg.Mesh.structgen(40, 36, 33, order=order) if mk == "struct"
            else cg.Mesh.jittered(30, 28, 26, 0.25, seed=3, permute=True, order=order))
    fields = _dev_fields(mesh, prec, 5)
    a = _run_fa(cg, mesh, prec, fields, False)
    b = _run_fa(cg, mesh, prec, fields, True)
    for k in ("grad", "mflux", "pb", "pbb", "sb"):
        assert torch.equal(a[k], b[k]), k
    assert torch.equal(a["loss"], b["loss"])


def test_rcm_bounds_bandwidth_of_permuted_mesh(cg, gpu):
    n = 24
    permuted = cg.Mesh.jittered(n, n, n, 0.25, seed=9, permute=True, order=cg.ORDER_NATIVE)
    rcm = cg.Mesh.jittered(n, n, n, 0.25, seed=9, permute=True, order=cg.ORDER_RCM)
    assert permuted.bandwidth > n ** 3 // 2
    assert rcm.bandwidth <= 2 * n * n
    native = cg.Mesh.structgen(n, n, n, order=cg.ORDER_NATIVE)
    assert native.bandwidth == n * n


@pytest.mark.parametrize("order", [2, 3])
def test_host_call_matches_oracle(cg, gpu, order):
    """The host-buffer forward+adjoint against the FP64 oracle."""
    ref = O.jitter(14, 12, 11, 0.25, seed=16, permute=True)
    mesh = cg.Mesh.from_arrays(ref, order=order)
    f = O.fields(ref, 17)
    gface = np.random.Generator(np.random.Philox(key=18)).standard_normal(ref["nFaces"])
    out = cg.forward_adjoint(mesh, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    _, g_ref, _ = O.gradient(ref, f["phi"], f["phiB"], 1)
    assert np.array_equal(out["grad"], g_ref)
    A = _adjoint_oracle(ref, f, gface)
    for k, v in A.items():
        e = errs(out[k], v)
        assert e["norm"] <= 1e-13 and e["rms"] <= 1e-13, (k, e)


@pytest.mark.parametrize("order", [1, 3])
def test_host_call_float_arrays_equal_double_arrays(cg, gpu, order):
    """The FP32 forward+adjoint through float host arrays
    (cupcfd_gpu_forward_adjoint_f32) returns the FP64-array call's results
    rounded to float, which are exact (the FP32 path's outputs are floats),
    and the same loss."""
    ref = O.jitter(14, 12, 11, 0.25, seed=18, permute=True)
    mesh = cg.Mesh.from_arrays(ref, order=order)
    f = O.fields(ref, 19)
    gface = np.random.Generator(np.random.Philox(key=20)).standard_normal(ref["nFaces"])
    ins = [as_f32(f[k]) for k in ("phi", "phiB", "den", "u", "v", "w")] + [as_f32(gface)]
    o64 = cg.forward_adjoint(mesh, cg.PREC_F32C, *ins)
    o32 = cg.forward_adjoint(mesh, cg.PREC_F32C, *[x.astype(np.float32) for x in ins])
    for k in ("grad", "massFlux", "phiBar", "phiBBar", "denBar", "uBar", "vBar", "wBar"):
        assert o32[k].dtype == np.float32, k
        assert np.array_equal(o32[k].astype(np.float64), o64[k]), k
    assert o32["loss"][0] == o64["loss"][0]


@pytest.mark.parametrize("order", [1, 3])
@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("mk", ["jitter", "poly"])
def test_host_call_equals_device_call(cg, gpu, order, prec, mk):
    """The host-buffer forward+adjoint (gradient, mass flux, loss and adjoint
    as separate launches, results copied back on a second stream while later
    inputs come in) returns what cupcfd_gpu_dev_forward_adjoint computes from
    the same values, bit for bit, the loss included; boundary faces' mass
    fluxes come back as zero."""
    import torch
    dev = torch.device("cuda:0")
    if mk == "jitter":
        ref = O.jitter(22, 20, 18, 0.25, seed=21, permute=True)
    else:
        ref = O.merge_cells(O.jitter(16, 15, 14, 0.25, seed=23, permute=True), 0.3, 24, max_cells=4)
    mesh = cg.Mesh.from_arrays(ref, order=order)
    f = O.fields(ref, 25)
    gface = np.random.Generator(np.random.Philox(key=26)).standard_normal(ref["nFaces"])
    cg.timing_read()
    cg.timing_enable(True)
    try:
        host = cg.forward_adjoint(mesh, prec, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
        ran = set(cg.timing_read())
    finally:
        cg.timing_enable(False)
    # the adjoint's two parts: the L2-prefetch kernels in FP32 on a tiled mesh
    # whose cell count allows whole 16-byte state ranges, else the plain
    # adjoint kernel
    if prec == cg.PREC_F32C and mesh.tiles and mesh.nCells % 4 == 0:
        assert {"k_gadj_f32_pf", "k_madj_f32_pf"} <= ran, sorted(ran)
    else:
        assert ("k_adj_f64" if prec == cg.PREC_F64 else "k_adj_f32") in ran, sorted(ran)
    c2o, f2o = mesh.numbering()
    nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
    dt = torch.float64 if prec == cg.PREC_F64 else torch.float32

    def T(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)

    st4 = np.stack([f[k][c2o] for k in ("den", "u", "v", "w")])
    state = T(st4) if prec == cg.PREC_F64 else T(st4.T)
    out = dict(grad=torch.full((3, nC), float("nan"), dtype=dt, device=dev),
               mf=torch.zeros(nF, dtype=dt, device=dev), pb=torch.full((nC,), float("nan"), dtype=dt, device=dev),
               pbb=torch.full((nB,), float("nan"), dtype=dt, device=dev), sb=torch.full_like(state, float("nan")),
               loss=torch.zeros(1, dtype=torch.float64, device=dev))
    s = torch.cuda.current_stream()
    cg.dev_forward_adjoint(mesh, prec, T(f["phi"][c2o]), T(f["phiB"]), state, T(gface[f2o]), out["grad"], out["mf"],
                           out["pb"], out["pbb"], out["sb"], out["loss"], stream=s)
    assert mesh.check_status(s) == cg.E_SUCCESS
    torch.cuda.synchronize()

    def to_ref(t, n2o):
        a = t.cpu().double().numpy()
        r = np.empty_like(a)
        r[..., n2o] = a
        return r

    def bits(a, b, what):
        a, b = np.ascontiguousarray(a, np.float64), np.ascontiguousarray(b, np.float64)
        assert a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64)), what

    bits(host["grad"], to_ref(out["grad"], c2o).T, "grad")
    inner = ref["faceCell2"] >= 0
    mf = to_ref(out["mf"], f2o)
    bits(host["massFlux"][inner], mf[inner], "massFlux")
    assert np.all(host["massFlux"][~inner] == 0.0)
    bits(host["phiBar"], to_ref(out["pb"], c2o), "phiBar")
    bits(host["phiBBar"], out["pbb"].cpu().double().numpy(), "phiBBar")
    sb = to_ref(out["sb"] if prec == cg.PREC_F64 else out["sb"].t(), c2o)
    for i, k in enumerate(("denBar", "uBar", "vBar", "wBar")):
        bits(host[k], sb[i], k)
    bits(host["loss"], out["loss"].cpu().numpy(), "loss")


def test_strided_vector_views_upload(cg, gpu):
    """Mesh creation from the vector arrays in every layout a caller can
    hand over (packed (n,3); the EuclideanVector layout (n,4) with the
    components after a pad slot; records whose components are not aligned
    to 8 bytes, 28-byte records with the components at byte 4): the same
    device geometry bit for bit."""
    import ctypes as C
    ref = O.jitter(9, 8, 7, 0.25, seed=31, permute=True)
    base = cg.Mesh.from_arrays(ref).geometry()
    padded = dict(ref)
    for k in ("faceNorm", "faceCenter", "cellCenter"):
        a = np.asarray(ref[k], np.float64).reshape(-1, 3)
        padded[k] = np.concatenate([np.full((len(a), 1), 7.5), a], 1)
    g4 = cg.Mesh.from_arrays(padded).geometry()
    for k in base:
        assert np.array_equal(base[k], g4[k]), k
    # 28-byte records, components at byte offset 4 (not 8-byte aligned)
    keep = {}

    def odd(a):
        a = np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1, 3))
        buf = np.zeros((len(a), 28), np.uint8)
        buf[:, 4:] = a.view(np.uint8).reshape(len(a), 24)
        keep[id(buf)] = buf
        return cg.Vec3View(buf.ctypes.data, 28, 4)

    v = cg.MeshView()
    v.nCells, v.nFaces, v.nBoundaries, v.real_size = ref["nCells"], ref["nFaces"], ref["nBnd"], 8
    arr = {k: np.ascontiguousarray(ref[k]) for k in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceArea",
                                                     "cellVolume")}
    v.faceCell1, v.faceCell2, v.faceBnd = (cg._p(arr[k]) for k in ("faceCell1", "faceCell2", "faceBnd"))
    v.faceLambda, v.faceArea, v.cellVolume = (cg._p(arr[k]) for k in ("faceLambda", "faceArea", "cellVolume"))
    v.faceNorm, v.faceCenter, v.cellCenter = odd(ref["faceNorm"]), odd(ref["faceCenter"]), odd(ref["cellCenter"])
    v.faceXpac = v.faceXnac = cg.Vec3View(None, 24, 0)
    h = C.c_void_p()
    o = cg.Mesh._opts(cg.ORDER_MORTON, (1 << cg.PREC_F64) | (1 << cg.PREC_F32C), -1)
    assert cg.lib().cupcfd_gpu_mesh_create(C.byref(v), C.byref(o), C.byref(h)) == cg.E_SUCCESS, cg.last_error()
    godd = cg.Mesh(h).geometry()
    for k in base:
        assert np.array_equal(base[k], godd[k]), k
    # overlapping records are refused
    v.faceNorm = cg.Vec3View(v.faceNorm.base, 28, 8)
    h2 = C.c_void_p()
    assert cg.lib().cupcfd_gpu_mesh_create(C.byref(v), C.byref(o), C.byref(h2)) == cg.E_CONFIG_INVALID_VALUE


def test_host_call_null_outputs(cg, gpu):
    """Outputs of the host forward+adjoint may be NULL: the others come back
    unchanged."""
    ref = O.jitter(12, 11, 10, 0.25, seed=41, permute=True)
    mesh = cg.Mesh.from_arrays(ref, order=cg.ORDER_OWNER)
    f = O.fields(ref, 42)
    gface = np.random.Generator(np.random.Philox(key=43)).standard_normal(ref["nFaces"])
    full = cg.forward_adjoint(mesh, cg.PREC_F32C, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    out = {k: np.full_like(v, np.nan) for k, v in full.items()}
    keep = ("phiBar", "uBar", "loss")
    rc = cg.lib().cupcfd_gpu_forward_adjoint(
        mesh.h, cg.PREC_F32C, *[cg._p(np.ascontiguousarray(f[k])) for k in ("phi", "phiB", "den", "u", "v", "w")],
        cg._p(gface), *[cg._p(out[k]) if k in keep else None for k in ("grad", "massFlux", "phiBar", "phiBBar", "denBar",
                                                                      "uBar", "vBar", "wBar", "loss")])
    assert rc == cg.E_SUCCESS, cg.last_error()
    for k in out:
        if k in keep:
            assert np.array_equal(out[k], full[k]), k
        else:
            assert np.all(np.isnan(out[k])), k


@pytest.mark.parametrize("mk", ["struct", "jitter"])
@pytest.mark.parametrize("ngrad", [1, 2, 3])
def test_gradient_float_instantiation_bit_exact(cg, gpu, mk, ngrad):
    """GradientPhiGaussDolfyn with T=float arrays and CUPCFD_PREC_F32REF
    against the reference's own T=float instantiation (compiled unchanged),
    on a mesh uploaded from the same float arrays: bit for bit, the
    non-orthogonal correction of later iterations included."""
    if O.load_ref() is None:
        pytest.skip("reference build absent")
    ref = O.structgen(11, 9, 8) if mk == "struct" else O.jitter(11, 9, 8, 0.25, seed=52, permute=True)
    m32 = dict(ref)
    for k in ("faceLambda", "faceArea", "faceNorm", "faceCenter", "cellCenter", "cellVolume"):
        m32[k] = np.ascontiguousarray(np.asarray(ref[k]), np.float32)
    f = O.fields(ref, 53)
    phi, phiB = f["phi"].astype(np.float32), f["phiB"].astype(np.float32)
    want, want_o = O.ref_gradient_f32(m32, phi, phiB, ngrad)
    mesh = cg.Mesh.from_arrays(m32, order=cg.ORDER_OWNER)
    n = ref["nCells"]
    g = np.full((n, 4), np.nan, np.float32)
    go = np.full((n, 4), np.nan, np.float32)
    rc = cg.GradientPhiGaussDolfyn(mesh, ngrad, phi, phiB, g, go, precision=cg.PREC_F32REF)
    assert rc == cg.E_SUCCESS, cg.last_error()
    assert np.array_equal(g[:, 1:].view(np.int32), want.view(np.int32))
    assert np.array_equal(go[:, 1:].view(np.int32), want_o.view(np.int32))
    # the precision exists for the gradient calls only
    out = cg.lib().cupcfd_gpu_forward_adjoint(mesh.h, cg.PREC_F32REF, *[None] * 16)
    assert out in (cg.E_NULL_PTR, cg.E_CONFIG_INVALID_VALUE)
