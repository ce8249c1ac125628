"""FluxMassDolfynBoundaryLoop1-5 and FluxMassDolfynRegionLoop on the GPU.

The host-buffer calls run the chain a solver step runs (inflow, area rate,
outlet fluxes, outflow per region, region factors, scaled outlet fluxes and
their su update) and every output is compared, bit for bit, with the
oracle, which is itself bit-identical to the reference's templates
(tests/test_oracle_vs_reference.py). The device-resident calls run the same
chain in the mesh's internal numbering, with every scalar left on the
device, and must give the same bits. Meshes: structured and jittered with
permuted numbering, six boundary regions (inlet, two outlets, symmetry,
wall, default) assigned at random, so that cells with several outlet faces
exercise the ordered su update; the large jittered mesh (112 x 104 x 96,
64,768 boundaries) takes the id-ordered sums through many staged passes.
"""
import numpy as np
import pytest

import oracle as O
from test_oracle_vs_reference import _with_regions

pytestmark = pytest.mark.gpu


def _setup(cg, kind, order):
    base = {"struct": lambda: O.structgen(20, 18, 16),
            "jitter": lambda: O.jitter(17, 15, 13, 0.25, seed=8, permute=True),
            "large": lambda: O.jitter(112, 104, 96, 0.25, seed=8, permute=True)}[kind]()
    m, splvl, rng = _with_regions(base, 41 if kind == "struct" else 42)
    mesh = cg.Mesh.from_arrays(m, order=order)
    assert mesh.set_regions(m["regionType"], m["regionUVW"], m["regionDen"], m["bndRegion"]) == cg.E_SUCCESS
    assert mesh.set_region_split(splvl) == cg.E_SUCCESS
    nF, nB, nC, nR = m["nFaces"], m["nBnd"], m["nCells"], m["nRegions"]
    d = dict(mf=rng.uniform(1e-6, 1e-2, nF) * rng.choice([-1.0, 1.0], nF),
             u=rng.uniform(1e-6, 1e-2, nB), v=rng.uniform(1e-6, 1e-2, nB), w=rng.uniform(1e-6, 1e-2, nB),
             den=rng.uniform(0.9, 1.1, nB), fr=rng.uniform(1e-6, 1e-2, nR), su=rng.standard_normal(nC))
    return m, splvl, mesh, d


def _oracle_chain(m, splvl, d, solve):
    flowin = O.boundary_loop1(m, d["mf"])
    ratearea = O.boundary_loop3(m, flowin)
    mf4, u4, v4, w4, flowout4 = O.boundary_loop4(m, splvl, d["mf"], d["u"], d["v"], d["w"], d["den"], ratearea)
    fr2, flowout2 = O.boundary_loop2(m, mf4, d["fr"])
    ff = O.region_loop(m, splvl, fr2, flowin)
    mf5, su5, u5, v5, w5, fo2 = O.boundary_loop5(m, mf4, d["su"], u4, v4, w4, 1.3, solve, ff, 0.25)
    return dict(flowin=flowin, ratearea=ratearea, mf4=mf4, u4=u4, v4=v4, w4=w4, flowout4=flowout4, fr2=fr2,
                flowout2=flowout2, ff=ff, mf5=mf5, su5=su5, u5=u5, v5=v5, w5=w5, fo2=fo2)


def _host_chain(cg, mesh, d, solve, f32=False):
    """The chain through the host-buffer calls; f32: float32 arrays (the
    reference's T = float instantiation)."""
    r = {}
    E = cg.E_SUCCESS
    rc, r["flowin"] = cg.FluxMassDolfynBoundaryLoop1(mesh, d["mf"].copy())
    assert rc == E
    rc, r["ratearea"] = cg.FluxMassDolfynBoundaryLoop3(mesh, r["flowin"], f32=f32)
    assert rc == E
    mf, u, v, w = d["mf"].copy(), d["u"].copy(), d["v"].copy(), d["w"].copy()
    rc, r["flowout4"] = cg.FluxMassDolfynBoundaryLoop4(mesh, mf, u, v, w, d["den"].copy(), r["ratearea"])
    assert rc == E
    r.update(mf4=mf.copy(), u4=u.copy(), v4=v.copy(), w4=w.copy())
    fr = d["fr"].copy()
    rc, r["flowout2"] = cg.FluxMassDolfynBoundaryLoop2(mesh, mf, fr)
    assert rc == E
    r["fr2"] = fr
    ff = np.full(len(fr), np.nan, fr.dtype)
    assert cg.FluxMassDolfynRegionLoop(mesh, ff, fr, r["flowin"]) == E
    r["ff"] = ff
    su = d["su"].copy()
    rc, r["fo2"] = cg.FluxMassDolfynBoundaryLoop5(mesh, mf, su, u, v, w, 1.3, solve, ff, 0.25)
    assert rc == E
    r.update(mf5=mf, su5=su, u5=u, v5=v, w5=w)
    return r


def test_many_regions_bit_exact(cg, gpu):
    """2,500 regions (more than one block of region sums: the region sums
    run in groups of 992): loops 1-5 and the region loop, and the momentum
    loop's boundary loop (wall shear onto each region's force tangent), bit
    for bit against the oracle."""
    base = O.jitter(30, 28, 26, 0.25, seed=12, permute=True)
    rng = np.random.Generator(np.random.Philox(key=43))
    nR = 2500
    m = dict(base)
    m["nRegions"] = nR
    m["regionType"] = rng.integers(0, 5, nR).astype(np.int32)
    m["regionUVW"] = rng.standard_normal(3 * nR)
    m["regionDen"] = rng.uniform(0.9, 1.1, nR)
    m["bndRegion"] = rng.integers(0, nR, m["nBnd"]).astype(np.int32)
    splvl = rng.uniform(0.2, 0.8, nR)
    mesh = cg.Mesh.from_arrays(m, order=3)
    assert mesh.set_regions(m["regionType"], m["regionUVW"], m["regionDen"], m["bndRegion"]) == cg.E_SUCCESS
    assert mesh.set_region_split(splvl) == cg.E_SUCCESS
    nF, nB, nC = m["nFaces"], m["nBnd"], m["nCells"]
    d = dict(mf=rng.uniform(1e-6, 1e-2, nF) * rng.choice([-1.0, 1.0], nF),
             u=rng.uniform(1e-6, 1e-2, nB), v=rng.uniform(1e-6, 1e-2, nB), w=rng.uniform(1e-6, 1e-2, nB),
             den=rng.uniform(0.9, 1.1, nB), fr=rng.uniform(1e-6, 1e-2, nR), su=rng.standard_normal(nC))
    want = _oracle_chain(m, splvl, d, (1, 1, 1))
    got = _host_chain(cg, mesh, d, (1, 1, 1))
    for k, v in want.items():
        assert np.array_equal(np.asarray(got[k]), np.asarray(v)), k
    # momentum loop's boundary loop on a shear the test sets
    shear = rng.standard_normal((nB, 3))
    ft0 = rng.standard_normal((nR, 3))
    mesh.boundary_shear(shear)
    mesh.region_force_tangent(nR, ft0)
    assert cg.FluxUVWDolfynBndsLoop1(mesh) == cg.E_SUCCESS
    assert np.array_equal(mesh.region_force_tangent(nR), O.uvw_bnds_loop1(m, shear, ft0))


@pytest.mark.parametrize("kind,order", [("struct", 2), ("jitter", 3), ("jitter", 0), ("large", 3)])
@pytest.mark.parametrize("solve", [(1, 1, 1), (0, 1, 0)])
def test_boundary_loops_bit_exact(cg, gpu, kind, order, solve):
    m, splvl, mesh, d = _setup(cg, kind, order)
    want = _oracle_chain(m, splvl, d, solve)
    got = _host_chain(cg, mesh, d, solve)
    for k, v in want.items():
        assert np.array_equal(np.asarray(got[k]), np.asarray(v)), k


@pytest.mark.parametrize("kind,order", [("struct", 2), ("jitter", 3)])
def test_device_loops_equal_host_loops(cg, gpu, kind, order):
    import torch
    dev = torch.device("cuda:0")
    m, splvl, mesh, d = _setup(cg, kind, order)
    solve = (1, 0, 1)
    host = _host_chain(cg, mesh, d, solve)
    c2o, f2o = mesh.numbering()

    def T(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    mf, su = T(d["mf"][f2o]), T(d["su"][c2o])
    u, v, w, den, fr = T(d["u"]), T(d["v"]), T(d["w"]), T(d["den"]), T(d["fr"])
    sc = torch.full((5,), np.nan, dtype=torch.float64, device=dev)      # flowin, ratearea, flowout4, flowout2, fo2
    ff = torch.full((m["nRegions"],), np.nan, dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream()
    cg.dev_boundary_loop1(mesh, mf, sc[0:1], stream=s)
    cg.dev_boundary_loop3(mesh, sc[0:1], sc[1:2], stream=s)
    cg.dev_boundary_loop4(mesh, mf, u, v, w, den, sc[1:2], sc[2:3], stream=s)
    mf4, u4 = mf.clone(), u.clone()
    cg.dev_boundary_loop2(mesh, mf, fr, sc[3:4], stream=s)
    cg.dev_region_loop(mesh, ff, fr, sc[0:1], stream=s)
    sc[4] = 0.25
    cg.dev_boundary_loop5(mesh, mf, su, u, v, w, 1.3, solve, ff, sc[4:5], stream=s)
    torch.cuda.synchronize()

    def H(t):
        return t.cpu().numpy()

    def to_ref(t, n2o):
        """internal -> reference numbering (internal i is reference n2o[i])"""
        a = H(t)
        out = np.empty_like(a)
        out[n2o] = a
        return out

    scal = H(sc)
    for k, x in (("flowin", scal[0]), ("ratearea", scal[1]), ("flowout4", scal[2]), ("flowout2", scal[3]),
                 ("fo2", scal[4])):
        assert x == host[k], k
    assert np.array_equal(to_ref(mf4, f2o), host["mf4"]) and np.array_equal(H(u4), host["u4"])
    assert np.array_equal(H(fr), host["fr2"]) and np.array_equal(H(ff), host["ff"])
    assert np.array_equal(to_ref(mf, f2o), host["mf5"]) and np.array_equal(to_ref(su, c2o), host["su5"])
    for k, t in (("u5", u), ("v5", v), ("w5", w)):
        assert np.array_equal(H(t), host[k]), k


@pytest.mark.parametrize("kind,order", [("struct", 2), ("jitter", 3), ("large", 0)])
def test_float_instantiation_bit_exact(cg, gpu, kind, order):
    """The _f32 calls (float32 host arrays) on a mesh made from float arrays
    against the reference's own T = float instantiation (compiled
    unchanged) on the same float arrays: the whole chain, every array and
    scalar bit for bit."""
    if O.load_ref() is None:
        pytest.skip("reference build absent")
    m, splvl, _, d = _setup(cg, kind, order)
    m32 = dict(m)
    for k in ("faceLambda", "faceArea", "faceNorm", "faceCenter", "faceXpac", "faceXnac", "cellCenter", "cellVolume",
              "regionUVW", "regionDen"):
        if m.get(k) is not None:
            m32[k] = np.ascontiguousarray(np.asarray(m[k]), np.float32)
    sp32 = splvl.astype(np.float32)
    mesh = cg.Mesh.from_arrays(m32, order=order)
    assert mesh.set_regions(m["regionType"], m32["regionUVW"].astype(np.float64),
                            m32["regionDen"].astype(np.float64), m["bndRegion"]) == cg.E_SUCCESS
    assert mesh.set_region_split(sp32.astype(np.float64)) == cg.E_SUCCESS
    d32 = {k: np.ascontiguousarray(v, np.float32) for k, v in d.items()}
    solve = (1, 0, 1)
    want = O.ref_boundary_chain_f32(m32, sp32, d32, 1.3, solve, 0.25)
    got = _host_chain(cg, mesh, d32, solve, f32=True)
    for k in ("flowin", "ratearea", "flowout4", "flowout2", "fo2"):
        assert np.float32(got[k]).view(np.int32) == np.float32(want[k]).view(np.int32), (k, got[k], want[k])
    for k in ("mf5", "su5", "u5", "v5", "w5", "fr2", "ff"):
        assert got[k].dtype == np.float32
        assert np.array_equal(got[k].view(np.int32), want[k].view(np.int32)), k
    assert want["flowin"] != 0 and want["fo2"] != 0.25


def test_boundary_loop_errors(cg, gpu):
    m, splvl, mesh, d = _setup(cg, "struct", 2)
    short = d["mf"][:-1].copy()
    assert cg.FluxMassDolfynBoundaryLoop1(mesh, short)[0] == cg.E_INVALID_INDEX
    assert cg.FluxMassDolfynBoundaryLoop2(mesh, d["mf"].copy(), d["fr"][:-1].copy())[0] == cg.E_INVALID_INDEX
    assert mesh.set_region_split(splvl[:-1]) == cg.E_ARRAY_SIZE_MISMATCH
    rc = cg.lib().cupcfd_gpu_flux_mass_dolfyn_boundary_loop3(mesh.h, 1.0, None)
    assert rc == cg.E_NULL_PTR
