"""The reference's real mesh class, built by the reference itself.

oracle/_ref/realmesh_dropin (tests/cpp/realmesh_dropin.cpp, `make -C oracle
realmesh`) builds CupCfdSoAMesh<int,double,int> the way a reference run does:
the CUP-CFD JSON configuration tests/cpp/realmesh.json read by
include/cupcfd_gpu/config.hpp, then the reference's own
MeshConfig::buildUnstructuredMesh -> PartitionerNaive ->
CupCfdSoAMesh::addData / finalize, compiled unchanged, on 2 and 4 ranks of
the in-process MPI stand-in (oracle/ref_mpi/mpi.h). The reference cannot
build a mesh on one rank (its BroadcastMPI returns E_NO_DATA for the empty
ghost list of DistributedAdjacencyList::finalize), so every case has at
least two ranks, as the reference's own mesh tests (4 ranks) do.

CPU: every rank's cellFaceMapCSRXAdj / Adj (owned and ghost cells) equals
the oracle's restatement of updateCellFaceMap on that rank's faces; the
ranks own every cell once; the configuration reader's errors.
GPU (marked gpu): the drop-in and the benchmark entry points on those real
meshes against the reference templates, bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "realmesh_dropin")
CFG = os.path.join(ROOT, "tests", "cpp", "realmesh.json")
need_bin = pytest.mark.skipif(not os.path.exists(BIN), reason="real-mesh program not built (needs the reference sources)")


def _read(path):
    b = open(path, "rb").read()
    off, out = 0, []
    while off < len(b):
        n = int(np.frombuffer(b, np.int64, 1, off)[0])
        off += 8
        out.append(np.frombuffer(b, np.int32, n, off).copy())
        off += 4 * n
    return out


@need_bin
@pytest.mark.parametrize("ranks", [2, 4])
def test_real_mesh_csr_matches_oracle(tmp_path, ranks):
    r = subprocess.run([BIN, "--dump", str(tmp_path), CFG, str(ranks)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.startswith("OK dump"), r.stdout + r.stderr
    owned = 0
    for k in range(ranks):
        head, c1, c2, bnd, xadj, adj = _read(os.path.join(tmp_path, f"rank{k}.bin"))
        nC, nO, nF, nB = (int(x) for x in head)
        assert len(c1) == len(c2) == len(bnd) == nF and len(xadj) == nC + 1
        rx, ra = O.cell_face_csr(dict(nCells=nC, nFaces=nF, faceCell1=c1, faceCell2=c2))
        assert np.array_equal(xadj, rx) and np.array_equal(adj, ra), f"rank {k}"
        assert np.array_equal(bnd >= 0, c2 < 0)
        owned += nO
    assert owned == 13 * 11 * 9


@need_bin
def test_configuration_errors(tmp_path):
    bad = tmp_path / "bad.json"
    bad.write_text('{"Mesh": {"MeshSource": ')
    r = subprocess.run([BIN, "--dump", str(tmp_path), str(bad), "2"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "configuration unreadable" in r.stdout
    nomesh = tmp_path / "nomesh.json"
    nomesh.write_text('{"Benchmarks": [{"BenchmarkKernels": {"BenchmarkName": "K", "Repetitions": 1}}]}')
    r = subprocess.run([BIN, "--dump", str(tmp_path), str(nomesh), "2"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "no MeshSourceStructGen mesh" in r.stdout
    nobench = tmp_path / "nobench.json"
    txt = open(CFG).read()
    nobench.write_text(txt[:txt.index('"Benchmarks"')].rstrip().rstrip(",") + "}")
    r = subprocess.run([BIN, "--dump", str(tmp_path), str(nobench), "2"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "no kernel benchmarks" in r.stdout


@pytest.mark.gpu
@need_bin
@pytest.mark.parametrize("ranks", [2, 4])
def test_real_mesh_dropin_and_benchmarks(gpu, ranks):
    r = subprocess.run([BIN, CFG, str(ranks)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK realmesh" in r.stdout, r.stdout
