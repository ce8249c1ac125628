"""Parity at the benchmark configurations' own sizes.

  config 2: 256^3 structured, against the oracle itself: the FP64 forward
            bit for bit and its adjoint within 1e-13; the FP32-compensated
            forward + adjoint against the oracle fed the same FP32-rounded
            inputs, every output within 1e-6 normwise and RMS, elementwise
            within 16 u sum|term| (forward) or the floored 5e-5 (adjoint).
  config 3: 192^3 jittered, cell and face numbering permuted: the FP64
            gradient and mass flux bit-identical to the oracle, the FP32
            path within the same normwise / RMS bounds and, element by
            element, within 16 u sum|term| (u = 2^-24).
  config 4: adjoint against central differences (eps = 1e-6, FP64, 64
            seeded directions, <= 1e-6 relative) on 128^3 structured and
            96^3 jittered meshes, and against the oracle's FP64 adjoint on
            the 96^3 mesh.

The finite differences are evaluated on the GPU with the FP64 forward. The
loss is quadratic in the inputs, so a central difference is exact up to
rounding; it is summed as L(x+ed) - L(x-ed) = sum_c V_c (g+ - g-).(g+ + g-)
+ sum_f g_f (m+ - m-), cell by cell, which keeps the rounding of a loss
of size ~1e4 out of a difference of size ~1e-5.
"""
import numpy as np
import pytest

import oracle as O
from test_gpu_parity import as_f32, assert_f32c, assert_incidences_match, errs, _adjoint_oracle, _loss_oracle

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _cell2_volume(cg, mesh):
    """faceCell2 and cellVolume in the mesh's internal numbering (only those
    two arrays are downloaded)."""
    c2 = np.empty(mesh.nFaces, np.int32)
    vol = np.empty(mesh.nCells)
    assert cg.lib().cupcfd_gpu_mesh_get_geometry(mesh.h, None, cg._p(c2), None, None, None, None, None, None,
                                                 cg._p(vol)) == cg.E_SUCCESS
    c2o, f2o = mesh.numbering()
    return c2[f2o], vol[c2o]


@pytest.fixture(scope="module")
def config2():
    """The 256^3 unit-cube mesh of the oracle with seeded fields and face
    weights in the reference's numbering (about 9 GB of host memory, 16 s)."""
    ref = O.structgen(256, 256, 256)
    f = O.fields(ref, 20261205)
    gface = np.random.Generator(np.random.Philox(key=20261211)).standard_normal(ref["nFaces"])
    return ref, f, gface


def test_config2_fp64_256_equals_oracle(cg, gpu, config2):
    """FP64 forward bit for bit, FP64 adjoint within 1e-13, against the
    oracle itself on the 256^3 benchmark mesh (host-buffer call)."""
    ref, f, gface = config2
    mesh = cg.Mesh.structgen(256, 256, 256, order=cg.ORDER_OWNER)
    out = cg.forward_adjoint(mesh, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    rc, g_ref, _ = O.gradient(ref, f["phi"], f["phiB"], 1)
    mf_ref = O.mass_plain(ref, f["den"], f["u"], f["v"], f["w"])
    inner = ref["faceCell2"] >= 0
    assert np.array_equal(out["grad"], g_ref)
    assert np.array_equal(out["massFlux"][inner], mf_ref[inner])
    for k, v in _adjoint_oracle(ref, f, gface).items():
        e = errs(out[k], v)
        assert e["norm"] <= 1e-13 and e["rms"] <= 1e-13, (k, e)
    mesh.close()


def test_config2_f32c_256_vs_oracle(cg, gpu, config2):
    """FP32-compensated forward + adjoint on the 256^3 benchmark mesh against
    the FP64 oracle fed the same FP32-rounded fields: every output (gradient,
    mass flux, dL/dphi, dL/dphi_b, dL/d(rho, u, v, w)) within 1e-6 normwise
    and RMS; gradient and mass flux element by element within
    16 u sum|term| (u = 2^-24, sum|term| from the oracle on absolute values),
    the adjoints within 5e-5 floored at 1e-2 rms; the loss within 1e-6."""
    ref, f, gface = config2
    mesh = cg.Mesh.structgen(256, 256, 256, order=cg.ORDER_OWNER)
    f32 = {k: as_f32(v) if isinstance(v, np.ndarray) and v.dtype == np.float64 else v for k, v in f.items()}
    g32 = as_f32(gface)
    out = cg.forward_adjoint(mesh, cg.PREC_F32C, f32["phi"], f32["phiB"], f32["den"], f32["u"], f32["v"], f32["w"],
                             g32)
    mesh.close()
    r32 = dict(ref)
    for k in ("faceNorm", "faceLambda"):
        r32[k] = as_f32(ref[k])
    rc, g_ref, _ = O.gradient(r32, f32["phi"], f32["phiB"], 1)
    mf_ref = O.mass_plain(r32, f32["den"], f32["u"], f32["v"], f32["w"])
    inner = ref["faceCell2"] >= 0
    for got, want, what in ((out["grad"], g_ref, "grad"), (out["massFlux"][inner], mf_ref[inner], "massFlux")):
        e = errs(got, want)
        assert e["norm"] <= 1e-6 and e["rms"] <= 1e-6, (what, e)
    ra = dict(r32)
    ra["faceNorm"] = np.abs(r32["faceNorm"])
    rc, g_abs, _ = O.gradient(ra, np.abs(f32["phi"]), np.abs(f32["phiB"]), 1)
    mf_abs = O.mass_plain(ra, np.abs(f32["den"]), np.abs(f32["u"]), np.abs(f32["v"]), np.abs(f32["w"]))
    u = 2.0 ** -24
    assert np.all(np.abs(out["grad"] - g_ref) <= 16 * u * g_abs), "gradient above 16 u sum|term|"
    assert np.all(np.abs(out["massFlux"][inner] - mf_ref[inner]) <= 16 * u * mf_abs[inner]), "mass flux above 16 u sum|term|"
    for k, v in _adjoint_oracle(r32, f32, g32).items():
        assert_f32c(out[k], v, k, elem=5e-5)
    L, _, _ = _loss_oracle(r32, f32, g32)
    assert abs(out["loss"][0] - L) <= 1e-6 * abs(L)


def test_config3_jittered_permuted_192(cg, gpu):
    ref = O.jitter(192, 192, 192, 0.25, seed=3, permute=True)
    mesh = cg.Mesh.jittered(192, 192, 192, 0.25, seed=3, permute=True, order=cg.ORDER_RCM)
    # connectivity: the reference-numbered CSR, and the RCM-renumbered lists
    # the kernels read, both bit for bit against the oracle's
    xadj, adj = mesh.cell_face_csr()
    rx, ra = O.cell_face_csr(ref)
    assert np.array_equal(xadj, rx) and np.array_equal(adj, ra)
    assert_incidences_match(mesh, ref)
    f = O.fields(ref, 20261206)
    rc, g_ref, _ = O.gradient(ref, f["phi"], f["phiB"], 1)
    mf_ref = O.mass_plain(ref, f["den"], f["u"], f["v"], f["w"])
    out = cg.forward_adjoint(mesh, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"],
                             np.zeros(ref["nFaces"]))
    assert np.array_equal(out["grad"], g_ref)
    inner = ref["faceCell2"] >= 0
    assert np.array_equal(out["massFlux"][inner], mf_ref[inner])
    # FP32 path against the FP64 oracle fed the same FP32-rounded fields and geometry
    f32 = {k: as_f32(v) if isinstance(v, np.ndarray) and v.dtype == np.float64 else v for k, v in f.items()}
    r32 = dict(ref)
    for k in ("faceNorm", "faceLambda"):
        r32[k] = as_f32(ref[k])
    rc, g32_ref, _ = O.gradient(r32, f32["phi"], f32["phiB"], 1)
    mf32_ref = O.mass_plain(r32, f32["den"], f32["u"], f32["v"], f32["w"])
    out = cg.forward_adjoint(mesh, cg.PREC_F32C, f32["phi"], f32["phiB"], f32["den"], f32["u"], f32["v"], f32["w"],
                             np.zeros(ref["nFaces"]))
    # Normwise and RMS bounds as on the small meshes. Elementwise, a
    # relative error floored at 1e-2 rms is a maximum over 7.1M cells and
    # 21M faces that grows with their number (1.3e-5 / 2.2e-5 here), so the
    # per-element check is the size-independent a-priori bound of a sum of
    # rounded terms: |got - ref| <= 16 u sum|term|, u = 2^-24, with sum|term|
    # from the oracle run on absolute values (all terms then add up).
    for got, ref_v, what in ((out["grad"], g32_ref, "gradient"), (out["massFlux"][inner], mf32_ref[inner], "mass")):
        e = errs(got, ref_v)
        assert e["norm"] <= 1e-6 and e["rms"] <= 1e-6, (what, e)
    ra = dict(r32)
    ra["faceNorm"] = np.abs(r32["faceNorm"])
    rc, g_abs, _ = O.gradient(ra, np.abs(f32["phi"]), np.abs(f32["phiB"]), 1)
    mf_abs = O.mass_plain(ra, np.abs(f32["den"]), np.abs(f32["u"]), np.abs(f32["v"]), np.abs(f32["w"]))
    u = 2.0 ** -24
    assert np.all(np.abs(out["grad"] - g32_ref) <= 16 * u * g_abs), "gradient above 16 u sum|term|"
    assert np.all(np.abs(out["massFlux"][inner] - mf32_ref[inner]) <= 16 * u * mf_abs[inner]), "mass flux above 16 u sum|term|"


def _fd_against_adjoint(cg, mesh, seed):
    """max over 64 directions of |FD - <grad L, d>| / |<grad L, d>|, FP64."""
    torch = _torch()
    dev = torch.device("cuda:0")
    nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
    c2, vol = _cell2_volume(cg, mesh)
    V = torch.from_numpy(vol).to(dev)
    inner = torch.from_numpy(c2 >= 0).to(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    dt = torch.float64
    phi = torch.rand(nC, generator=g, device=dev, dtype=dt) * 2 - 1
    phiB = torch.rand(nB, generator=g, device=dev, dtype=dt) * 2 - 1
    st = torch.randn(4, nC, generator=g, device=dev, dtype=dt)
    st[0] = 0.9 + 0.2 * torch.rand(nC, generator=g, device=dev, dtype=dt)
    gface = torch.randn(nF, generator=g, device=dev, dtype=dt)
    s = torch.cuda.current_stream()
    grad = torch.empty(3, nC, dtype=dt, device=dev)
    mf = torch.zeros(nF, dtype=dt, device=dev)
    pb, pbb = torch.empty(nC, dtype=dt, device=dev), torch.empty(nB, dtype=dt, device=dev)
    sb = torch.empty(4, nC, dtype=dt, device=dev)
    cg.dev_forward_adjoint(mesh, cg.PREC_F64, phi, phiB, st, gface, grad, mf, pb, pbb, sb, stream=s)

    def fwd(p, pB, sv):
        gr = torch.empty(3, nC, dtype=dt, device=dev)
        m = torch.zeros(nF, dtype=dt, device=dev)
        cg.dev_forward(mesh, cg.PREC_F64, p, pB, sv, gr, m, stream=s)
        return gr, m

    eps, worst = 1e-6, 0.0
    for _ in range(64):
        d_phi = torch.randn(nC, generator=g, device=dev, dtype=dt)
        d_phiB = torch.randn(nB, generator=g, device=dev, dtype=dt)
        d_st = torch.randn(4, nC, generator=g, device=dev, dtype=dt)
        gp, mp = fwd(phi + eps * d_phi, phiB + eps * d_phiB, st + eps * d_st)
        gm, mm = fwd(phi - eps * d_phi, phiB - eps * d_phiB, st - eps * d_st)
        dL = float(torch.sum(V * torch.sum((gp - gm) * (gp + gm), 0)) + torch.sum(gface[inner] * (mp - mm)[inner]))
        fd = dL / (2 * eps)
        ad = float(torch.dot(pb, d_phi) + torch.dot(pbb, d_phiB) + torch.sum(sb * d_st))
        worst = max(worst, abs(fd - ad) / max(abs(ad), 1e-300))
    assert mesh.check_status(s) == cg.E_SUCCESS
    return worst


def test_config4_adjoint_central_differences_128(cg, gpu):
    mesh = cg.Mesh.structgen(128, 128, 128, order=cg.ORDER_OWNER)
    assert _fd_against_adjoint(cg, mesh, 20261207) <= 1e-6


def test_config4_adjoint_96_jittered(cg, gpu):
    ref = O.jitter(96, 96, 96, 0.25, seed=4, permute=True)
    mesh = cg.Mesh.jittered(96, 96, 96, 0.25, seed=4, permute=True, order=cg.ORDER_RCM)
    assert _fd_against_adjoint(cg, mesh, 20261208) <= 1e-6
    # and against the oracle's FP64 adjoint (reference numbering, host call)
    f = O.fields(ref, 20261209)
    gface = np.random.Generator(np.random.Philox(key=20261210)).standard_normal(ref["nFaces"])
    out = cg.forward_adjoint(mesh, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    for k, v in _adjoint_oracle(ref, f, gface).items():
        e = errs(out[k], v)
        assert e["norm"] <= 1e-13 and e["rms"] <= 1e-13, (k, e)
