"""Mesh ingest from the reference's HDF5 mesh files (MeshHDF5Source) by the
library's own HDF5 reader.

CPU:
* the reference's fixture tests/geometry/mesh/data/MeshHDF5.hdf5 against
  the expectations of the reference's MeshHDF5SourceTests.cpp
  (tests/golden/meshhdf5source_golden.json; the file is read from the
  reference tree, so these cases run where it is present): counts, cell and
  boundary labels, boundary flags, cell volumes and face counts, and the
  face lambdas and normals the reference's disabled cases state (the file
  stores them as float32, so they are compared as float32 values);
* files written by tests/h5write.py (float64 meshes in the same layout)
  read back bit for bit;
* files written by the library's own writer read back bit for bit, hold
  /cell/nfaces, /cell/cface and /bnd/face as MeshHDF5Source reads them, and
  read as the same mesh as the test writer's; the reference fixture's own
  connectivity datasets agree with the connectivity read from its faces;
* missing, foreign, truncated and inconsistent files return the reference's
  error codes, for reading and for writing.
GPU: a written file loads as the same device mesh as the arrays it came
from, regions and boundary distances included, and the face loops give the
same bits on it; a device mesh saved with save_hdf5 loads back the same.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from h5write import mesh_hdf5_bytes

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "meshhdf5source_golden.json")))


def _reference_root():
    """The reference checkout: CUPCFD_REFERENCE, else the one oracle/Makefile
    compiled oracle/_ref from (empty when neither exists)."""
    env = os.environ.get("CUPCFD_REFERENCE")
    if env:
        return env
    rec = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "reference_root.txt")
    return open(rec).read().strip() if os.path.exists(rec) else ""


FIXTURE = os.path.join(_reference_root(), GOLD["fixture"]) if _reference_root() else ""
need_fixture = pytest.mark.skipif(not (FIXTURE and os.path.exists(FIXTURE)), reason="reference fixture absent")


def _case(name):
    return next(c for c in GOLD["cases"] if c["name"] == name)


def _arr(name, key):
    return _case(name)["arrays"][key]["values"]


@need_fixture
def test_reference_fixture_matches_reference_expectations(cg):
    m = cg.hdf5_mesh_read(FIXTURE)
    assert m["nCells"] == _case("getCellCount_test1")["scalars"]["cells"]
    assert m["nFaces"] == _case("getFaceCount_test1")["scalars"]["faces"]
    assert m["nBnd"] == _case("getBoundaryCount_test1")["scalars"]["boundaries"]
    assert m["nRegions"] == _case("getRegionCount_test1")["scalars"]["regions"]
    # face -> cell labels (1-based; cell2 -1 on boundary faces)
    labels = np.array(_arr("getFaceCell1Labels_test1", "faceLabels")) - 1
    assert np.array_equal(m["faceCell1"][labels] + 1, _arr("getFaceCell1Labels_test1", "cellLabelsCmp"))
    c2 = m["faceCell2"][labels]
    assert np.array_equal(np.where(c2 >= 0, c2 + 1, -1), _arr("getFaceCell2Labels_test1", "cellLabelsCmp"))
    isb = np.array(_arr("getFaceIsBoundary_test1", "isBoundaryCmp"), bool)
    assert np.array_equal(m["faceCell2"][np.array(_arr("getFaceIsBoundary_test1", "faceLabels")) - 1] < 0, isb)
    bl = np.array(_arr("getFaceBoundaryLabels_test1", "faceLabels")) - 1
    assert np.array_equal(m["faceBnd"][bl] + 1, _arr("getFaceBoundaryLabels_test1", "boundaryLabelsCmp"))
    # cell volumes and face counts of cells 1, 3, 4
    cl = np.array(_arr("getCellVolume_test1", "nLabels")) - 1
    vol = _arr("getCellVolume_test1", "volCmp")[:len(cl)]
    assert np.array_equal(m["cellVolume"][cl], vol)
    xadj, _ = O.cell_face_csr(m)
    cl = np.array(_arr("getCellNFaces_test1", "nLabels")) - 1
    assert np.array_equal(np.diff(xadj)[cl], _arr("getCellNFaces_test1", "nFacesCmp"))
    assert np.diff(xadj).max() == _case("getMaxFaceCount_test1")["scalars"]["maxFaceCount"]
    # lambda and normals, as the file stores them (float32)
    f32 = lambda v: np.asarray(v, np.float32).astype(np.float64)
    assert np.array_equal(m["faceLambda"], f32(_arr("getFaceLambda2_test1", "faceLambdaCmp")))
    nrm = np.stack([_arr("getFaceNormal_test1", k) for k in ("normalCmpX", "normalCmpY", "normalCmpZ")], 1)
    assert np.array_equal(m["faceNorm"], f32(nrm))


@need_fixture
def test_reference_fixture_truncated_and_foreign(cg, tmp_path):
    data = open(FIXTURE, "rb").read()
    for cut in (64, 500, 3000, len(data) - 200):
        p = tmp_path / f"cut{cut}.h5"
        p.write_bytes(data[:cut])
        with pytest.raises(cg.CupcfdError) as e:
            cg.hdf5_mesh_read(str(p))
        assert e.value.code == cg.E_INVALID_FILE_FORMAT, cut


@pytest.mark.parametrize("kind", ["struct", "jitter", "poly"])
def test_written_mesh_reads_back(cg, tmp_path, kind):
    from test_oracle_vs_reference import _with_regions
    base = {"struct": lambda: O.structgen(7, 6, 5),
            "jitter": lambda: O.jitter(7, 6, 5, 0.25, seed=3, permute=True),
            "poly": lambda: O.merge_cells(O.jitter(8, 7, 6, 0.25, seed=4, permute=True), 0.3, 5, max_cells=4)}[kind]()
    m, _, rng = _with_regions(base, 70)
    dist = rng.uniform(0.01, 0.2, m["nBnd"])
    p = tmp_path / "m.h5"
    p.write_bytes(mesh_hdf5_bytes(m, dist))
    r = cg.hdf5_mesh_read(str(p))
    for k in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceArea", "faceNorm", "faceCenter", "cellCenter",
              "cellVolume", "bndRegion"):
        assert np.array_equal(r[k], np.asarray(m[k]).reshape(r[k].shape)), k
    assert np.array_equal(r["bndDistance"], dist)
    assert (r["nCells"], r["nFaces"], r["nBnd"], r["nRegions"]) == (m["nCells"], m["nFaces"], m["nBnd"], m["nRegions"])


def test_error_codes(cg, tmp_path):
    with pytest.raises(cg.CupcfdError) as e:
        cg.hdf5_mesh_read(str(tmp_path / "absent.h5"))
    assert e.value.code == cg.E_FILE_MISSING
    p = tmp_path / "text.h5"
    p.write_bytes(b"not an HDF5 file" * 20)
    with pytest.raises(cg.CupcfdError) as e:
        cg.hdf5_mesh_read(str(p))
    assert e.value.code == cg.E_INVALID_FILE_FORMAT
    # a face pointing past the cells
    m = O.structgen(3, 3, 3)
    bad = dict(m)
    bad["faceCell1"] = m["faceCell1"].copy()
    bad["faceCell1"][5] = m["nCells"] + 3
    p.write_bytes(mesh_hdf5_bytes(bad))
    with pytest.raises(cg.CupcfdError) as e:
        cg.hdf5_mesh_read(str(p))
    assert e.value.code == cg.E_INVALID_INDEX
    # counts that do not match the datasets
    p.write_bytes(mesh_hdf5_bytes(m))
    rc = cg.lib().cupcfd_gpu_hdf5_mesh_read(os.fsencode(str(p)), m["nCells"] + 1, m["nFaces"], m["nBnd"],
                                           *[None] * 11)
    assert rc == cg.E_ARRAY_SIZE_MISMATCH


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 3])
def test_load_hdf5_equals_arrays(cg, gpu, tmp_path, order):
    from test_gpu_uvw import _check, _host
    from test_oracle_vs_reference import uvw_case
    m, rng = uvw_case("jitter", 71, "outlet")
    dist = rng.uniform(0.01, 0.2, m["nBnd"])
    p = tmp_path / "m.h5"
    p.write_bytes(mesh_hdf5_bytes(m, dist))
    loaded = cg.Mesh.load_hdf5(str(p), order=order)
    ref = cg.Mesh.from_arrays(m, order=order)
    ga, gb = loaded.geometry(), ref.geometry()
    for k in ga:
        assert np.array_equal(ga[k], gb[k]), k
    f = O.fields(m, 72)
    gface = np.random.Generator(np.random.Philox(key=73)).standard_normal(m["nFaces"])
    a = cg.forward_adjoint(loaded, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    b = cg.forward_adjoint(ref, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    # regions come in as default regions (MeshHDF5Source): the momentum loop
    # sees the boundaries' distances, and no inlet, outlet or wall
    m0 = dict(m)
    m0["regionType"] = np.zeros_like(m["regionType"])
    fu = O.uvw_fields(m0, 74)
    _check(_host(cg, loaded, fu), O.uvw_face_loop1(m0, fu, None, dist))


# ---------------------------------------------------------------------------
# the library's writer
# ---------------------------------------------------------------------------
def _written(cg, tmp_path, kind, seed=80):
    from test_oracle_vs_reference import _with_regions
    base = {"struct": lambda: O.structgen(7, 6, 5),
            "jitter": lambda: O.jitter(7, 6, 5, 0.25, seed=3, permute=True),
            "poly": lambda: O.merge_cells(O.jitter(8, 7, 6, 0.25, seed=4, permute=True), 0.3, 5, max_cells=4)}[kind]()
    m, _, rng = _with_regions(base, seed)
    dist = rng.uniform(0.01, 0.2, m["nBnd"])
    p = str(tmp_path / f"lib_{kind}.h5")
    cg.hdf5_mesh_write(p, m, dist)
    return m, dist, p


@pytest.mark.parametrize("kind", ["struct", "jitter", "poly"])
def test_library_writer_round_trip(cg, tmp_path, kind):
    """A file the library writes reads back bit for bit, and holds the
    connectivity datasets MeshHDF5Source reads: /cell/nfaces, /cell/cface
    (each cell's faces ascending, 1-based, 0-padded) and /bnd/face."""
    m, dist, p = _written(cg, tmp_path, kind)
    r = cg.hdf5_mesh_read(p)
    for k in ("faceCell1", "faceCell2", "faceBnd", "faceLambda", "faceArea", "faceNorm", "faceCenter", "cellCenter",
              "cellVolume", "bndRegion"):
        assert np.array_equal(r[k], np.asarray(m[k]).reshape(r[k].shape)), k
    assert np.array_equal(r["bndDistance"], dist)
    assert (r["nCells"], r["nFaces"], r["nBnd"], r["nRegions"]) == (m["nCells"], m["nFaces"], m["nBnd"], m["nRegions"])
    xadj, adj = O.cell_face_csr(m)
    nf = np.diff(xadj)
    assert np.array_equal(cg.hdf5_dataset(p, "/cell/nfaces"), nf)
    cface = cg.hdf5_dataset(p, "/cell/cface")
    assert cface.shape == (m["nCells"], nf.max())
    for c in range(m["nCells"]):
        assert np.array_equal(cface[c, :nf[c]] - 1, adj[xadj[c]:xadj[c + 1]]), c
        assert np.all(cface[c, nf[c]:] == 0)
    bface = cg.hdf5_dataset(p, "/bnd/face").astype(np.int64) - 1
    assert np.array_equal(np.asarray(m["faceBnd"])[bface], np.arange(m["nBnd"]))
    assert np.array_equal(cg.hdf5_dataset(p, "/face/cell2"), np.where(m["faceCell2"] >= 0, m["faceCell2"] + 1, 0))


def test_library_writer_equals_test_writer(cg, tmp_path):
    """The library's file and the test-only writer's file read as the same
    mesh."""
    m, dist, p = _written(cg, tmp_path, "jitter", 81)
    q = tmp_path / "py.h5"
    q.write_bytes(mesh_hdf5_bytes(m, dist))
    a, b = cg.hdf5_mesh_read(p), cg.hdf5_mesh_read(str(q))
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


def test_library_writer_errors(cg, tmp_path):
    m = O.structgen(3, 3, 3)
    bad = dict(m)
    bad["faceCell2"] = m["faceCell2"].copy()
    bad["faceCell2"][4] = m["nCells"]
    with pytest.raises(cg.CupcfdError) as e:
        cg.hdf5_mesh_write(str(tmp_path / "a.h5"), bad)
    assert e.value.code == cg.E_INVALID_INDEX
    dup = dict(m)
    dup["faceBnd"] = m["faceBnd"].copy()
    b = np.flatnonzero(m["faceCell2"] < 0)
    dup["faceBnd"][b[1]] = dup["faceBnd"][b[0]]
    with pytest.raises(cg.CupcfdError) as e:
        cg.hdf5_mesh_write(str(tmp_path / "b.h5"), dup)
    assert e.value.code == cg.E_INVALID_INDEX
    with pytest.raises(cg.CupcfdError) as e:
        cg.hdf5_mesh_write(str(tmp_path / "no_such_dir" / "c.h5"), m)
    assert e.value.code == cg.E_FILE_MISSING
    with pytest.raises(cg.CupcfdError) as e:
        cg.hdf5_dataset(str(tmp_path / "absent.h5"), "/cell/vol")
    assert e.value.code == cg.E_FILE_MISSING


@need_fixture
def test_reference_fixture_connectivity_datasets(cg):
    """The reference fixture's own /cell/nfaces, /cell/cface and /bnd/face
    agree with the connectivity the library reads from /face/cell1, cell2
    and bnd."""
    m = cg.hdf5_mesh_read(FIXTURE)
    xadj, adj = O.cell_face_csr(m)
    nf = cg.hdf5_dataset(FIXTURE, "/cell/nfaces").astype(np.int64)
    assert np.array_equal(nf, np.diff(xadj))
    cface = cg.hdf5_dataset(FIXTURE, "/cell/cface").astype(np.int64)
    for c in range(m["nCells"]):
        assert sorted(cface[c, :nf[c]] - 1) == sorted(adj[xadj[c]:xadj[c + 1]]), c
    bface = cg.hdf5_dataset(FIXTURE, "/bnd/face").astype(np.int64) - 1
    assert np.array_equal(m["faceBnd"][bface], np.arange(m["nBnd"]))


@pytest.mark.gpu
def test_save_hdf5_load_hdf5(cg, gpu, tmp_path):
    """A device mesh written with save_hdf5 loads back as the same mesh (its
    boundaries' regions and distances included) and gives the same bits."""
    from test_oracle_vs_reference import uvw_case
    m, rng = uvw_case("jitter", 82, "outlet")
    dist = rng.uniform(0.01, 0.2, m["nBnd"])
    mesh = cg.Mesh.from_arrays(m, order=3)
    assert mesh.set_regions(m["regionType"], m["regionUVW"], m["regionDen"], m["bndRegion"]) == cg.E_SUCCESS
    assert mesh.set_boundary_distance(dist) == cg.E_SUCCESS
    p = str(tmp_path / "dev.h5")
    mesh.save_hdf5(p)
    r = cg.hdf5_mesh_read(p)
    assert np.array_equal(r["bndRegion"], m["bndRegion"]) and np.array_equal(r["bndDistance"], dist)
    loaded = cg.Mesh.load_hdf5(p, order=3)
    ga, gb = loaded.geometry(), mesh.geometry()
    for k in ga:
        assert np.array_equal(ga[k], gb[k]), k
    f = O.fields(m, 83)
    gface = np.random.Generator(np.random.Philox(key=84)).standard_normal(m["nFaces"])
    a = cg.forward_adjoint(loaded, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    b = cg.forward_adjoint(mesh, cg.PREC_F64, f["phi"], f["phiB"], f["den"], f["u"], f["v"], f["w"], gface)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
