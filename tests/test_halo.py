"""Meshes split across ranks (cup-cfd_b200/halo.py), on CPU.

* partition_naive follows the reference's PartitionerNaive assignment
  (PartitionerNaive.cpp:97-128), vectors worked out from that formula, and
  refuses the sizes where that formula puts cells past the last part.
* Local meshes: every owned cell's faces are local and in ascending global
  face id; each rank's send list to a peer is that peer's ghost range from
  it, cell for cell.
* The decomposition keeps the single-rank arithmetic: the oracle's gradient
  and full mass-flux loop on each local mesh, ghosts filled with their
  owners' values, equal the global ones bit for bit on owned cells / faces.
* The transfer: two gloo ranks exchange ghost values with halo.transfer
  (batched isend / irecv) and receive exactly their ghosts' global values.
"""
import os
import socket

import numpy as np
import pytest

import oracle as O
from conftest import load_cupcfd


def _halo():
    load_cupcfd()
    import cupcfd_b200.halo as H
    return H


def test_partition_naive_matches_reference_formula():
    H = _halo()
    assert H.partition_naive(10, 3).tolist() == [0, 0, 0, 0, 1, 1, 1, 2, 2, 2]
    assert H.partition_naive(11, 3).tolist() == [0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2]
    assert H.partition_naive(12, 4).tolist() == [0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3]
    p = H.partition_naive(1000, 7)
    assert np.all(np.diff(p) >= 0) and np.bincount(p).tolist() == [143, 143, 143, 143, 143, 143, 142]
    with pytest.raises(ValueError):
        H.partition_naive(7, 4)     # remainder 3 against part size 1: cells past part 3
    with pytest.raises(ValueError):
        H.partition_naive(3, 4)


def _case(kind, nparts):
    H = _halo()
    if kind == "struct":
        m = O.structgen(12, 10, 9)
        part = H.partition_naive(m["nCells"], nparts)
    elif kind == "jitter":
        m = O.jitter(11, 10, 9, 0.25, seed=4, permute=True)
        rng = np.random.default_rng(3)
        part = H.partition_blocks(rng.permutation(m["nCells"]) if nparts == 1 else
                                  np.argsort(m["cellCenter"][:, 0] + 0.37 * m["cellCenter"][:, 1]), nparts)
    else:
        m = O.merge_cells(O.jitter(10, 9, 8, 0.25, seed=6, permute=True), 0.35, 3, max_cells=4)
        part = H.partition_blocks(np.argsort(m["cellCenter"][:, 2]), nparts)
    return H, m, part


@pytest.mark.parametrize("kind", ["struct", "jitter", "poly"])
@pytest.mark.parametrize("nparts", [2, 3, 5])
def test_local_meshes_and_exchange_lists(kind, nparts):
    H, m, part = _case(kind, nparts)
    locs = [H.local_mesh(m, part, r) for r in range(nparts)]
    gx, ga = O.cell_face_csr(m)
    assert sum(l["nOwned"] for l in locs) == m["nCells"]
    for l in locs:
        owned = l["cells"][:l["nOwned"]]
        assert np.all(part[owned] == l["rank"]) and np.all(np.diff(owned) > 0)
        lx, la = O.cell_face_csr(l)
        for i, c in enumerate(owned):
            got = l["faces"][la[lx[i]:lx[i + 1]]]
            assert np.array_equal(got, ga[gx[c]:gx[c + 1]]), (l["rank"], c)
        ghosts = l["cells"][l["nOwned"]:]
        assert not np.any(part[ghosts] == l["rank"])
        for p, (lo, hi) in l["recv"].items():
            sent = locs[p]["cells"][locs[p]["send"][l["rank"]]]
            assert np.array_equal(sent, l["cells"][lo:hi]), (p, l["rank"])
        for p in l["send"]:
            assert l["rank"] in locs[p]["recv"]
        assert np.array_equal(l["bndRegion"], m["bndRegion"][l["bnds"]])


def _fill_ghosts(l, glob):
    """A field on a local mesh: owned values, ghosts as exchanged (the global
    values at the ghosts), taken from the global field."""
    return np.ascontiguousarray(glob[l["cells"]])


@pytest.mark.parametrize("kind", ["jitter", "poly"])
def test_sharded_oracle_equals_single_rank(kind):
    """The oracle's kernels on each local mesh equal the global run on the
    cells / faces the rank owns: the decomposition changes no rounding."""
    H, m, part = _case(kind, 3)
    from test_oracle_vs_reference import _with_regions
    m, _, rng = _with_regions(m, 44)
    f = O.fields(m, 45, full=True)
    f["massFlux"] = rng.standard_normal(m["nFaces"])
    # nGradient = 1: later iterations read the neighbours' previous gradients,
    # which on ghost cells need an exchange between iterations (the kernel,
    # like the reference's, does none)
    rc, g, go = O.gradient(m, f["phi"], f["phiB"], 1)
    rc, want = O.flux_mass_face_loop(m, f)
    for r in range(3):
        l = H.local_mesh(m, part, r)
        nO = l["nOwned"]
        fl = {k: (_fill_ghosts(l, v) if isinstance(v, np.ndarray) and len(v) == m["nCells"] else v) for k, v in f.items()}
        fl["phiB"] = np.ascontiguousarray(f["phiB"][l["bnds"]])
        for k in ("denB", "teB", "edB", "visB", "tB"):
            fl[k] = np.ascontiguousarray(f[k][l["bnds"]])
        fl["massFlux"] = np.ascontiguousarray(f["massFlux"][l["faces"]])
        fl["rface"] = np.ascontiguousarray(f["rface"].reshape(-1, 2)[l["faces"]].reshape(-1))
        rc, gl, gol = O.gradient(l, fl["phi"], fl["phiB"], 1)
        assert np.array_equal(gl[:nO], g[l["cells"][:nO]]) and np.array_equal(gol[:nO], go[l["cells"][:nO]])
        rc, got = O.flux_mass_face_loop(l, fl)
        own_f = part[m["faceCell1"][l["faces"]]] == r
        assert np.array_equal(got["massFlux"][own_f], want["massFlux"][l["faces"][own_f]])
        assert np.array_equal(got["rface"].reshape(-1, 2)[own_f], want["rface"].reshape(-1, 2)[l["faces"][own_f]])
        assert np.array_equal(got["su"][:nO], want["su"][l["cells"][:nO]])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    try:
        import torch
        import torch.distributed as dist
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world)
        H, m, part = _case("poly", world)
        l = H.local_mesh(m, part, rank)
        field = np.arange(m["nCells"] * 3, dtype=np.float64).reshape(3, -1) * 1.5 + 0.25   # 3 components
        peers, send, recv, s_off, r_off = H.exchange_plan(l)
        local = field[:, l["cells"]].copy()
        local[:, l["nOwned"]:] = np.nan
        sendbuf = torch.from_numpy(np.ascontiguousarray(local[:, send].T).reshape(-1))   # element-major
        recvbuf = torch.full((len(recv) * 3,), float("nan"), dtype=torch.float64)
        H.transfer(peers, s_off, r_off, sendbuf, recvbuf, 3)
        local[:, recv] = recvbuf.numpy().reshape(-1, 3).T
        ok = np.array_equal(local, field[:, l["cells"]])
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, bool(ok), len(recv)))
    except Exception as ex:  # reported to the parent
        q.put((rank, repr(ex), 0))


def test_two_gloo_ranks_exchange_ghosts():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert sorted(r[0] for r in res) == [0, 1]
    for rank, ok, n in res:
        assert ok is True, (rank, ok)
        assert n > 0
