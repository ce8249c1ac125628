"""Pins the oracle's structured-mesh restatement to the reference's own golden
vectors (tests/geometry/mesh/implementation/source/MeshStructGenSourceTests.cpp,
extracted into tests/golden/meshstructgen_golden.json by
tests/golden/make_golden.py). CPU only."""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "meshstructgen_golden.json")
with open(GOLDEN) as fh:
    CASES = json.load(fh)["cases"]

# Cases that exercise the MPI partition graph (four ranks each holding a
# slice); the one-GPU path has no partitioner, so they have nothing to pin.
SKIP = {"buildDistributedAdjacencyList1_test1", "buildDistributedAdjacencyList2_test1",
        "buildDistributedAdjacencyList2_test2", "getRegionName_test1"}


def _mesh(case):
    c = case["ctor"]
    nx, ny, nz = int(c[0]), int(c[1]), int(c[2])
    return nx, ny, nz, O.structgen(nx, ny, nz, bounds=tuple(c[3:9]), with_vertices=True)


@pytest.mark.parametrize("case", [c for c in CASES if c["name"] not in SKIP], ids=lambda c: c["name"])
def test_golden_case(case):
    nx, ny, nz, m = _mesh(case)
    A, P, S = case["arrays"], case["points"], case["scalars"]
    meth = case["method"]
    nc, nf, nb, nv = O.counts(nx, ny, nz)
    if meth == "getCellLabels":
        assert A["cmp"] == A["indices"]          # labels are the 0-based indices
    elif meth == "getCellCount":
        assert nc == S["cellCount"]
    elif meth == "getFaceCount":
        assert nf == S["faceCount"] == m["nFaces"]
    elif meth == "getBoundaryCount":
        assert nb == S["boundaryCount"] == int(np.count_nonzero(m["faceBnd"] >= 0))
    elif meth == "getRegionCount":
        assert m["nRegions"] == S["regionCount"]
    elif meth == "getVertexCount":
        assert nv == S["vertexCount"] == len(m["vertCoords"])
    elif meth == "getMaxFaceCount":
        xadj, _ = O.cell_face_csr(m)
        assert np.diff(xadj).max() == S["maxFaceCount"]
    elif meth == "getMaxVertexCount":
        assert m["faceVert"].shape[1] == S["maxVertexCount"]
    elif meth == "getCellNFaces":
        xadj, _ = O.cell_face_csr(m)
        assert np.diff(xadj)[A["cellLabels"]].tolist() == A["cmp"]
    elif meth == "getCellCenter":
        got = m["cellCenter"][A["cellLabels"]]
        assert np.array_equal(got, np.array(P["cmp"]))
    elif meth == "getCellFaceLabels":
        xadj, adj = O.structgen_cell_face_labels(nx, ny, nz)
        assert xadj.tolist() == A["cmpIndices"]
        assert adj.tolist() == A["cmpData"]
    elif meth == "getFaceIsBoundary":
        assert (m["faceBnd"][A["faceLabels"]] >= 0).astype(int).tolist() == A["cmp"]
    elif meth in ("getFaceNVertices", "getBoundaryNVertices"):
        assert all(v == 4 for v in A["cmp"])
        assert m["faceVert"].shape[1] == 4
    elif meth == "getFaceBoundaryLabels":
        got = m["faceBnd"][A["faceLabels"]]
        if case["expect_status"] == "E_ERROR":
            assert (got < 0).any()                # an interior face in the list is an error
        else:
            assert got.tolist() == A["cmp"]
    elif meth == "getFaceCell1Labels":
        assert m["faceCell1"][A["faceLabels"]].tolist() == A["cmp"]
    elif meth == "getFaceCell2Labels":
        assert m["faceCell2"][A["faceLabels"]].tolist() == A["cmp"]
    elif meth == "getFaceVerticesLabelsCSR":
        fv = m["faceVert"][A["faceLabels"]]
        assert (np.arange(len(fv) + 1) * 4).tolist() == A["cmpIndices"]
        assert fv.ravel().tolist() == A["cmpData"]
    elif meth == "getVertexCoords":
        assert np.array_equal(m["vertCoords"][A["vertexLabels"]], np.array(P["cmp"]))
    elif meth == "getBoundaryFaceLabels":
        bface = np.empty(nb, np.int64)
        isb = m["faceBnd"] >= 0
        bface[m["faceBnd"][isb]] = np.nonzero(isb)[0]
        assert bface[A["boundaryLabels"]].tolist() == A["cmp"]
    elif meth == "getBoundaryRegionLabels":
        assert m["bndRegion"][A["boundaryLabels"]].tolist() == A["cmp"]
    elif meth == "getBoundaryVerticesLabelsCSR":
        bface = np.empty(nb, np.int64)
        isb = m["faceBnd"] >= 0
        bface[m["faceBnd"][isb]] = np.nonzero(isb)[0]
        fv = m["faceVert"][bface[A["boundaryLabels"]]]
        assert (np.arange(len(fv) + 1) * 4).tolist() == A["cmpIndices"]
        assert fv.ravel().tolist() == A["cmpData"]
    else:
        pytest.fail(f"unhandled golden case {case['name']} ({meth})")


def test_all_golden_cases_known():
    handled = {c["name"] for c in CASES} - SKIP
    assert len(handled) >= 20


def test_csr_is_sorted_source_cell_faces():
    """updateCellFaceMap's CSR equals the generator's per-cell face labels
    sorted ascending (CupCfdSoAMesh.cpp:549-668 on a one-rank mesh)."""
    for dims in [(2, 3, 4), (5, 4, 3), (1, 1, 1), (7, 1, 2)]:
        m = O.structgen(*dims)
        xadj, adj = O.cell_face_csr(m)
        sx, sa = O.structgen_cell_face_labels(*dims)
        assert np.array_equal(xadj, sx)
        for c in range(len(sx) - 1):
            assert np.array_equal(adj[sx[c]:sx[c + 1]], np.sort(sa[sx[c]:sx[c + 1]]))
