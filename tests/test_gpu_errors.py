"""Error behaviour of the C ABI: bad inputs return the reference's eCodes
values (never a trap), and the context stays usable afterwards."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _mesh():
    return O.structgen(4, 3, 2)


@pytest.mark.parametrize("bad", ["cell1_oob", "cell2_oob", "cell2_eq_cell1", "bnd_on_interior", "bnd_oob", "bnd_twice"])
def test_invalid_connectivity_is_rejected(cg, gpu, bad):
    m = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in _mesh().items()}
    interior = np.nonzero(m["faceCell2"] >= 0)[0]
    boundary = np.nonzero(m["faceCell2"] < 0)[0]
    if bad == "cell1_oob":
        m["faceCell1"][interior[3]] = m["nCells"]
    elif bad == "cell2_oob":
        m["faceCell2"][interior[2]] = -7
    elif bad == "cell2_eq_cell1":
        m["faceCell2"][interior[0]] = m["faceCell1"][interior[0]]
    elif bad == "bnd_on_interior":
        m["faceBnd"][interior[1]] = 0
    elif bad == "bnd_oob":
        m["faceBnd"][boundary[0]] = m["nBnd"]
    elif bad == "bnd_twice":
        m["faceBnd"][boundary[1]] = m["faceBnd"][boundary[0]]
    rc, mesh = cg.Mesh.from_arrays(m, return_code=True)
    assert rc == cg.E_INVALID_INDEX and mesh is None
    assert "invalid connectivity" in cg.last_error()
    # the context is still usable
    ok = cg.Mesh.from_arrays(_mesh())
    assert ok.nCells == 24


def test_empty_mesh_rejected(cg, gpu):
    m = dict(_mesh())
    m["nCells"] = 0
    rc, mesh = cg.Mesh.from_arrays(m, return_code=True)
    assert rc == cg.E_ARRAY_SIZE_MISMATCH


def test_short_arrays_are_index_errors(cg, gpu):
    ref = _mesh()
    mesh = cg.Mesh.from_arrays(ref)
    f = O.fields(ref, 1)
    n = ref["nCells"]
    g, go = np.empty((n, 3)), np.empty((n, 3))
    assert cg.GradientPhiGaussDolfyn(mesh, 1, f["phi"][:-1], f["phiB"], g, go) == cg.E_INVALID_INDEX
    assert cg.GradientPhiGaussDolfyn(mesh, 1, f["phi"], f["phiB"][:-1], g, go) == cg.E_INVALID_INDEX
    assert cg.GradientPhiGaussDolfyn(mesh, 1, f["phi"], f["phiB"], g[:-1], go[:-1]) == cg.E_INVALID_INDEX
    assert cg.GradientPhiGaussDolfyn(mesh, 1, f["phi"], f["phiB"], g, go) == cg.E_SUCCESS


def test_precision_not_built_is_config_error(cg, gpu):
    ref = _mesh()
    mesh = cg.Mesh.from_arrays(ref, precisions=1 << cg.PREC_F32C)
    f = O.fields(ref, 1)
    n = ref["nCells"]
    g, go = np.empty((n, 3)), np.empty((n, 3))
    assert cg.GradientPhiGaussDolfyn(mesh, 1, f["phi"], f["phiB"], g, go, precision=cg.PREC_F64) == cg.E_CONFIG_INVALID_VALUE
    assert cg.GradientPhiGaussDolfyn(mesh, 1, f["phi"], f["phiB"], g, go, precision=cg.PREC_F32C) == cg.E_SUCCESS
    assert cg.GradientPhiGaussDolfyn(mesh, 1, f["phi"], f["phiB"], g, go, precision=7) == cg.E_CONFIG_INVALID_VALUE
    assert cg.GradientPhiGaussDolfyn(mesh, 1, f["phi"], f["phiB"], g, go, precision=cg.PREC_F32C, sign_mode=5) == cg.E_CONFIG_INVALID_VALUE


def test_bad_regions_rejected(cg, gpu):
    ref = _mesh()
    mesh = cg.Mesh.from_arrays(ref)
    nb = ref["nBnd"]
    assert mesh.set_regions([0, 1], np.zeros((2, 3)), np.ones(2), np.full(nb, 2, np.int32)) == cg.E_INVALID_INDEX
    assert mesh.set_regions([0, 9], np.zeros((2, 3)), np.ones(2), np.zeros(nb, np.int32)) == cg.E_CONFIG_INVALID_VALUE
    assert mesh.set_regions([0, 1], np.zeros((2, 3)), np.ones(2), np.zeros(nb - 1, np.int32)) == cg.E_ARRAY_SIZE_MISMATCH
    assert mesh.set_regions([0, 1], np.zeros((2, 3)), np.ones(2), np.ones(nb, np.int32)) == cg.E_SUCCESS
