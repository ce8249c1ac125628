"""Polyhedral meshes on the GPU: cells of 6 to 26 faces (hexahedra merged
across removed faces, oracle.merge_cells), so the cells of a 32-cell slice
have different face counts and the SELL-32 lists take their per-slice
widths (no common width), cells need several entry chunks, and tiles hold
different numbers of entries and faces. Every path is checked against the
oracle (itself bit-identical to the reference on these meshes,
tests/test_oracle_vs_reference.py): FP64 bit for bit, FP32-compensated
within the error bounds of the hexahedral tests, and the forward+adjoint
variants (the one forward+adjoint call, the separate forward and adjoint
calls, the host call) against each other bit for bit.
"""
import numpy as np
import pytest

import oracle as O
from test_gpu_parity import _adjoint_oracle, _dev_fields, _mass_case, _run_fa, as_f32, assert_f32c, errs, vec4
from test_gpu_uvw import _check, _host
from test_oracle_vs_reference import _with_regions

pytestmark = pytest.mark.gpu

ORDERS = [0, 1, 2, 3]


def _poly(max_cells=6, dims=(9, 8, 7), seed=5, frac=0.4):
    m = O.merge_cells(O.jitter(*dims, 0.25, seed=seed, permute=True), frac, 11, max_cells=max_cells)
    deg = np.diff(O.cell_face_csr(m)[0])
    assert deg.min() == 6 and deg.max() >= 14
    return m


@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("max_cells", [3, 6])
def test_mesh_and_gradient_bit_exact(cg, gpu, order, max_cells):
    m = _poly(max_cells)
    mesh = cg.Mesh.from_arrays(m, order=order)
    assert mesh.maxCellFaces == int(np.diff(O.cell_face_csr(m)[0]).max())
    xadj, adj = mesh.cell_face_csr()
    rx, ra = O.cell_face_csr(m)
    assert np.array_equal(xadj, rx) and np.array_equal(adj, ra)
    f = O.fields(m, 3)
    for ng in (1, 2, 3):
        rc, g_ref, go_ref = O.gradient(m, f["phi"], f["phiB"], ng)
        g, go = vec4(m["nCells"]), vec4(m["nCells"])
        assert cg.GradientPhiGaussDolfyn(mesh, ng, f["phi"], f["phiB"], g, go) == cg.E_SUCCESS
        assert np.array_equal(g[:, 1:], g_ref) and np.array_equal(go[:, 1:], go_ref), ng


@pytest.mark.parametrize("order", [1, 3])
def test_mass_flux_with_regions_bit_exact(cg, gpu, order):
    m, splvl, rng = _with_regions(_poly(), 93)
    mesh = cg.Mesh.from_arrays(m, order=order)
    assert mesh.set_regions(m["regionType"], m["regionUVW"], m["regionDen"], m["bndRegion"]) == cg.E_SUCCESS
    f = O.fields(m, 31, full=True)
    f["massFlux"] = rng.standard_normal(m["nFaces"])
    f["solveTurbEnergy"] = f["solveEnthalpy"] = True
    f["icinl"], f["icsym"] = 3, 1   # the counters _mass_case starts from
    rc, want = O.flux_mass_face_loop(m, f)
    rc2, got = _mass_case(cg, mesh, m, f)
    assert rc == rc2 == cg.E_SUCCESS
    for k in ("massFlux", "su", "rface", "denB", "teB", "edB", "visB", "tB"):
        assert np.array_equal(got[k], want[k]), k
    for k in ("icinl", "icout", "icsym", "icwal"):
        assert got[k] == want[k], k


@pytest.mark.parametrize("order", [1, 2])
def test_forward_adjoint_host_call(cg, gpu, order):
    """FP64 against the oracle's adjoint; FP32 within the hexahedral bounds."""
    m = _poly()
    mesh = cg.Mesh.from_arrays(m, order=order)
    f = O.fields(m, 7)
    gface = np.random.Generator(np.random.Philox(key=8)).standard_normal(m["nFaces"])
    out = cg.forward_adjoint(mesh, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    rc, g_ref, _ = O.gradient(m, f["phi"], f["phiB"], 1)
    assert np.array_equal(out["grad"], g_ref)
    for k, v in _adjoint_oracle(m, f, gface).items():
        e = errs(out[k], v)
        assert e["norm"] <= 1e-13 and e["rms"] <= 1e-13, (k, e)
    f32 = {k: as_f32(v) if isinstance(v, np.ndarray) and v.dtype == np.float64 else v for k, v in f.items()}
    r32 = dict(m)
    for k in ("faceNorm", "faceLambda"):
        r32[k] = as_f32(m[k])
    g32 = as_f32(gface)
    out = cg.forward_adjoint(mesh, cg.PREC_F32C, f32["phi"], f32["phiB"], f32["den"], f32["u"], f32["v"], f32["w"], g32)
    rc, g_ref, _ = O.gradient(r32, f32["phi"], f32["phiB"], 1)
    assert_f32c(out["grad"], g_ref, "gradient")
    for k, v in _adjoint_oracle(r32, f32, g32).items():
        assert_f32c(out[k], v, k, elem=5e-5)


@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("prec", [0, 1])
def test_forward_adjoint_equals_separate_calls(cg, gpu, order, prec):
    """The forward+adjoint call and the separate forward and adjoint calls
    give the same bits on ragged slices and tiles."""
    import torch
    m = _poly(6, dims=(24, 22, 20), frac=0.3)
    mesh = cg.Mesh.from_arrays(m, order=order)
    fields = _dev_fields(mesh, prec, 5)
    a = _run_fa(cg, mesh, prec, fields, False)
    b = _run_fa(cg, mesh, prec, fields, True)
    for k in ("grad", "mflux", "pb", "pbb", "sb"):
        assert torch.equal(a[k], b[k]), k


@pytest.mark.parametrize("order", [1, 3])
def test_momentum_and_boundary_loops_bit_exact(cg, gpu, order):
    m, splvl, rng = _with_regions(_poly(), 94)
    m["bndRegion"][m["faceBnd"][0]] = 2
    rl, bd = rng.uniform(0.1, 2.0, m["nFaces"]), rng.uniform(0.01, 0.2, m["nBnd"])
    mesh = cg.Mesh.from_arrays(m, order=order)
    assert mesh.set_regions(m["regionType"], m["regionUVW"], m["regionDen"], m["bndRegion"]) == cg.E_SUCCESS
    assert mesh.set_region_split(splvl) == cg.E_SUCCESS
    assert mesh.set_face_rlencos(rl) == cg.E_SUCCESS and mesh.set_boundary_distance(bd) == cg.E_SUCCESS
    f = O.uvw_fields(m, 95)
    _check(_host(cg, mesh, f), O.uvw_face_loop1(m, f, rl, bd))
    mf = rng.uniform(1e-6, 1e-2, m["nFaces"]) * rng.choice([-1.0, 1.0], m["nFaces"])
    rc, flowin = cg.FluxMassDolfynBoundaryLoop1(mesh, mf.copy())
    assert rc == cg.E_SUCCESS and flowin == O.boundary_loop1(m, mf)
