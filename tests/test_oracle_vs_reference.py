"""Validates the plain-C oracle against the reference's own code, compiled
unchanged from its sources into oracle/_ref/libcupcfd_ref.so (make -C oracle
ref). Skipped where that build is absent. CPU only."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.skipif(O.load_ref() is None, reason="reference build absent (make -C oracle ref)")

DIMS = [(2, 3, 4), (5, 4, 3), (16, 16, 16), (1, 1, 1), (9, 2, 5)]
BOUNDS = [(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), (-1.0, 1.0, -1.0, 2.0, 0.0, 2.0), (0.0, 3.0, -0.5, 0.25, 1.0, 1.7)]


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("bounds", BOUNDS)
def test_structgen_geometry_bit_exact(dims, bounds):
    a = O.structgen(*dims, bounds=bounds, with_vertices=True)
    b = O.ref_structgen(*dims, bounds=bounds, with_vertices=True)
    for k in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceNorm", "faceCenter", "faceArea", "cellCenter",
              "faceVert", "vertCoords"):
        assert np.array_equal(a[k], b[k]), k
    # volume: exact box volume vs the reference's five-tetrahedron Heron sum,
    # whose own rounding reaches ~1e-14 relative on stretched cells
    rel = np.abs(a["cellVolume"] - b["cellVolume"]) / np.abs(b["cellVolume"])
    assert rel.max() <= 2e-14


@pytest.mark.parametrize("dims", DIMS[:3])
def test_csr_matches_source(dims):
    b = O.ref_structgen(*dims)
    xadj, adj = O.cell_face_csr(b)
    sx, sa = b["srcCellFaceXAdj"], b["srcCellFaceAdj"]
    assert np.array_equal(xadj, sx)
    for c in range(len(sx) - 1):
        assert np.array_equal(adj[sx[c]:sx[c + 1]], np.sort(sa[sx[c]:sx[c + 1]]))


@pytest.mark.parametrize("dims", [(2, 3, 4), (8, 8, 8), (5, 4, 3)])
@pytest.mark.parametrize("ngrad", [0, 1, 2, 3])
def test_gradient_bit_exact(dims, ngrad):
    m = O.ref_structgen(*dims)
    f = O.fields(m, 11, full=True)
    rc, g, go = O.gradient(m, f["phi"], f["phiB"], ngrad)
    R = O.RefKernels(m)
    rc2, g2, go2, _ = R.gradient(f["phi"], f["phiB"], ngrad)
    assert rc == rc2 == O.E_SUCCESS
    if ngrad > 0:
        assert np.array_equal(g, g2)
    assert np.array_equal(go, go2)


@pytest.mark.parametrize("full", [False, True])
@pytest.mark.parametrize("regions", [False, True])
def test_mass_flux_bit_exact(full, regions):
    m = O.ref_structgen(6, 5, 4)
    if regions:
        m = dict(m)
        m["nRegions"] = 5
        m["regionType"] = np.array([0, 1, 2, 3, 4], np.int32)
        rng = np.random.default_rng(3)
        m["regionUVW"] = rng.standard_normal((5, 3))
        m["regionDen"] = rng.uniform(0.5, 1.5, 5)
        m["bndRegion"] = rng.integers(0, 5, m["nBnd"]).astype(np.int32)
    f = O.fields(m, 5, full=full)
    f["solveTurbEnergy"] = f["solveTurbDiss"] = f["solveEnthalpy"] = True
    rc, out = O.flux_mass_face_loop(m, f)
    R = O.RefKernels(m)
    rc2, out2, _ = R.flux_mass(f)
    assert rc == rc2 == O.E_SUCCESS
    for k in ("massFlux", "su", "rface", "denB", "teB", "edB", "visB", "tB"):
        assert np.array_equal(out[k], out2[k]), k
    for k in ("icinl", "icout", "icsym", "icwal"):
        assert out[k] == out2[k]


def test_jittered_mesh_through_reference_kernels():
    """The reference kernels accept the jittered + permuted mesh arrays
    (as they would from MeshHDF5Source) and agree with the oracle bit for bit."""
    m = O.jitter(6, 5, 7, 0.25, seed=4, permute=True)
    f = O.fields(m, 9, full=True)
    rc, g, go = O.gradient(m, f["phi"], f["phiB"], 2)
    R = O.RefKernels(m)
    rc2, g2, go2, _ = R.gradient(f["phi"], f["phiB"], 2)
    assert rc == rc2 == O.E_SUCCESS and np.array_equal(g, g2)
    rc, out = O.flux_mass_face_loop(m, f)
    rc2, out2, _ = R.flux_mass(f)
    assert np.array_equal(out["massFlux"], out2["massFlux"]) and np.array_equal(out["rface"], out2["rface"])


def test_error_codes_match_reference_enum():
    ref = O.load_ref()
    assert ref.ref_ecode_success() == O.E_SUCCESS == 95
    assert ref.ref_ecode_invalid_index() == O.E_INVALID_INDEX == 68
    assert ref.ref_ecode_array_size_mismatch() == O.E_ARRAY_SIZE_MISMATCH == 25
    assert ref.ref_ecode_error() == O.E_ERROR == 98
    assert ref.ref_ecode_null_ptr() == 99
    assert ref.ref_ecode_not_implemented() == 109
    assert ref.ref_ecode_file_missing() == 10
    assert ref.ref_ecode_invalid_file_format() == 105
    assert ref.ref_ecode_config_opt_not_found() == 92
    # EuclideanVector<T,3> carries a vptr: 32-byte (double) / 24-byte (float) stride, components at +8
    assert ref.ref_sizeof_euclidean_vector_f64() == 32
    assert ref.ref_sizeof_euclidean_vector_f32() == 24
    assert ref.ref_offsetof_cmp_f64() == 8


def _with_regions(m, seed):
    """Six regions (default, inlet, two outlets, symmetry, wall), boundaries
    assigned at random, random split levels."""
    rng = np.random.Generator(np.random.Philox(key=seed))
    m = dict(m)
    m["nRegions"] = 6
    m["regionType"] = np.array([0, 1, 2, 3, 4, 2], np.int32)
    m["regionUVW"] = rng.standard_normal(18)
    m["regionDen"] = rng.uniform(0.9, 1.1, 6)
    m["bndRegion"] = rng.integers(0, 6, m["nBnd"]).astype(np.int32)
    splvl = rng.uniform(0.2, 0.8, 6)
    return m, splvl, rng


@pytest.mark.parametrize("mk", ["struct", "jitter"])
def test_boundary_and_region_loops_bit_exact(mk):
    """FluxMassDolfynBoundaryLoop1-5 and FluxMassDolfynRegionLoop: the C
    restatement against the reference templates, every output bit for bit."""
    base = O.structgen(9, 7, 8) if mk == "struct" else O.jitter(9, 8, 7, 0.25, seed=4, permute=True)
    m, splvl, rng = _with_regions(base, 31 if mk == "struct" else 32)
    R = O.RefKernels(m).boundary_loops(splvl)
    nF, nB, nC, nR = m["nFaces"], m["nBnd"], m["nCells"], m["nRegions"]
    mf = rng.uniform(1e-6, 1e-2, nF) * rng.choice([-1.0, 1.0], nF)
    assert O.boundary_loop1(m, mf) == R.boundary_loop1(mf)
    fr0 = rng.uniform(1e-6, 1e-2, nR)
    fa, oa = O.boundary_loop2(m, mf, fr0)
    fb, ob = R.boundary_loop2(mf, fr0)
    assert np.array_equal(fa, fb) and oa == ob
    assert O.boundary_loop3(m, 1.1) == R.boundary_loop3(1.1)
    u, v, w, den = (rng.uniform(1e-6, 1e-2, nB) for _ in range(4))
    a4 = O.boundary_loop4(m, splvl, mf, u, v, w, den, -0.37)
    b4 = R.boundary_loop4(mf, u, v, w, den, -0.37)
    for x, y in zip(a4, b4):
        assert np.array_equal(x, y)
    su = rng.standard_normal(nC)
    ff = O.region_loop(m, splvl, fa, 0.7)
    assert np.array_equal(ff, R.region_loop(fa, 0.7))
    for solve in ((1, 1, 1), (1, 0, 1)):
        a5 = O.boundary_loop5(m, a4[0], su, u, v, w, 1.3, solve, ff, 0.25)
        b5 = R.boundary_loop5(a4[0], su, u, v, w, 1.3, solve, ff, 0.25)
        for x, y in zip(a5, b5):
            assert np.array_equal(x, y)
    # the outlet cells with several boundary faces are where su's order shows
    bf = np.full(nB, -1)
    inner = m["faceBnd"] > -1
    bf[m["faceBnd"][inner]] = np.nonzero(inner)[0]
    outlet = m["regionType"][m["bndRegion"]] == 2
    cells = m["faceCell1"][bf[outlet]]
    assert len(cells) > len(np.unique(cells))


def uvw_case(mk, seed, first="outlet"):
    """A mesh whose face 0 is a boundary face, regions at random with that
    face's boundary set to an inlet or outlet: the carried uFace / visFace the
    reference reads (UVWKernels.ipp:74-75) are then defined from face 0 on."""
    base = O.structgen(9, 7, 8) if mk == "struct" else O.jitter(9, 8, 7, 0.25, seed=5, permute=True)
    m, _, rng = _with_regions(base, seed)
    assert m["faceBnd"][0] >= 0
    m["bndRegion"][m["faceBnd"][0]] = 2 if first == "outlet" else 1
    return m, rng


def assert_same_bits(got, want, keys):
    for k in keys:
        a, b = np.asarray(got[k]), np.asarray(want[k])
        assert a.shape == b.shape, k
        assert np.array_equal(a.view(np.int64) if a.dtype == np.float64 else a,
                              b.view(np.int64) if b.dtype == np.float64 else b), k


@pytest.mark.parametrize("mk", ["struct", "jitter"])
@pytest.mark.parametrize("first", ["outlet", "inlet"])
@pytest.mark.parametrize("geom", ["zero", "set"])
def test_uvw_face_loop1_bit_exact(mk, first, geom):
    """FluxUVWDolfynFaceLoop1, RegionLoop1 and BndsLoop1: the C restatement
    against the reference templates, every output bit for bit. With zero
    boundary distances (what MeshSource-built meshes hold) the symmetry and
    wall branches divide by zero, and the infinities and NaNs must agree too."""
    m, rng = uvw_case(mk, 60 + (mk == "jitter"), first)
    f = O.uvw_fields(m, 61)
    rl = bd = None
    if geom == "set":
        rl = rng.uniform(0.1, 2.0, m["nFaces"])
        bd = rng.uniform(0.01, 0.2, m["nBnd"])
    R = O.RefKernels(m).uvw_geometry(rl, bd)
    rc, want, _ = R.uvw_face_loop1(f)
    assert rc == O.E_SUCCESS
    got = O.uvw_face_loop1(m, f, rl, bd)
    assert_same_bits(got, want, O.UVW_INOUT + ("shear",))
    if geom == "set":
        for k in ("su", "sv", "sw", "au", "av", "aw", "uB", "shear"):
            assert np.all(np.isfinite(got[k])), k
    # the branches all ran: outlets clamped negative fluxes, walls set shear
    bt = m["regionType"][m["bndRegion"]]
    bfaces = np.flatnonzero(m["faceBnd"] >= 0)
    out_f = bfaces[bt[m["faceBnd"][bfaces]] == 2]
    assert np.all(got["massFlux"][out_f] > 0) and np.any(f["massFlux"][out_f] < 0)
    if geom == "set":
        assert np.any(got["shear"][bt == 4] != 0)
    # region force tangents: zeroed, then the wall shears summed in boundary order
    R.uvw_state(force_tangent=np.full((m["nRegions"], 3), 7.0))
    ft0 = R.uvw_region_loop1()
    assert np.array_equal(ft0, O.uvw_region_loop1(m)) and not ft0.any()
    ft1 = R.uvw_bnds_loop1()
    assert_same_bits({"ft": O.uvw_bnds_loop1(m, got["shear"], ft0)}, {"ft": ft1}, ("ft",))


@pytest.mark.parametrize("mk", ["struct", "jitter"])
@pytest.mark.parametrize("first", ["outlet", "inlet"])
@pytest.mark.parametrize("geom", ["zero", "set"])
def test_uvw_loops_float_instantiation_bit_exact(mk, first, geom):
    """The momentum loops of the reference's T=float instantiation (face
    loop, region loop, boundary loop): the C float restatement against the
    reference's own float build, every output bit for bit, infinities and
    NaNs of the zero-distance case included."""
    m, rng = uvw_case(mk, 70 + (mk == "jitter"), first)
    f = O.uvw_fields(m, 71)
    rl = bd = None
    if geom == "set":
        rl = rng.uniform(0.1, 2.0, m["nFaces"])
        bd = rng.uniform(0.01, 0.2, m["nBnd"])
    want = O.ref_uvw_loops_f32(m, f, rl, bd)
    got = O.uvw_loops_f32(m, f, rl, bd)
    for k in O.UVW_INOUT + ("shear", "forceTangent"):
        a, b = np.asarray(got[k]), np.asarray(want[k])
        assert a.dtype == b.dtype == np.float32 and a.shape == b.shape, k
        assert np.array_equal(a.view(np.int32), b.view(np.int32)), k
    if geom == "set":
        bt = m["regionType"][m["bndRegion"]]
        assert np.any(got["shear"][bt == 4] != 0) and np.all(np.isfinite(got["su"]))


@pytest.mark.parametrize("max_cells", [3, 6])
def test_polyhedral_mesh_bit_exact(max_cells):
    """Cells of 6 to 26 faces (hexahedra merged across removed faces): the
    gradient, the full mass-flux loop with regions, the boundary loops and
    the momentum loop agree with the reference templates bit for bit."""
    m = O.merge_cells(O.jitter(9, 8, 7, 0.25, seed=5, permute=True), 0.4, 11, max_cells=max_cells)
    m, splvl, rng = _with_regions(m, 90 + max_cells)
    assert m["faceBnd"][0] >= 0
    m["bndRegion"][m["faceBnd"][0]] = 2
    deg = np.diff(O.cell_face_csr(m)[0])
    assert deg.min() == 6 and deg.max() >= 14
    f = O.fields(m, 91, full=True)
    f["massFlux"] = rng.standard_normal(m["nFaces"])
    R = O.RefKernels(m)
    for ng in (1, 2):
        rc, g, go, _ = R.gradient(f["phi"], f["phiB"], ng)
        rc2, g2, go2 = O.gradient(m, f["phi"], f["phiB"], ng)
        assert rc == rc2 == O.E_SUCCESS and np.array_equal(g, g2) and np.array_equal(go, go2)
    rc, want, _ = R.flux_mass(f)
    rc2, got = O.flux_mass_face_loop(m, f)
    assert rc == rc2 == O.E_SUCCESS
    for k in ("massFlux", "su", "rface", "denB"):
        assert np.array_equal(got[k], want[k]), k
    R.boundary_loops(splvl)
    mf = rng.uniform(1e-6, 1e-2, m["nFaces"])
    assert O.boundary_loop1(m, mf) == R.boundary_loop1(mf)
    fu = O.uvw_fields(m, 92)
    rl, bd = rng.uniform(0.1, 2.0, m["nFaces"]), rng.uniform(0.01, 0.2, m["nBnd"])
    rc, want, _ = R.uvw_geometry(rl, bd).uvw_face_loop1(fu)
    assert_same_bits(O.uvw_face_loop1(m, fu, rl, bd), want, O.UVW_INOUT + ("shear",))
