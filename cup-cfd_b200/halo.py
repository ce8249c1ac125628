"""Meshes split across ranks: cell partitioning, local meshes with ghost
cells, and the halo exchange of ghost-cell values.

Replaces, for this path, the reference's decomposition machinery:
  * PartitionerNaive::partition (src/partitioner/implementation/component/
    PartitionerNaive.cpp:59-140): contiguous blocks of cells in label order,
    the same assignment formula (``partition_naive``);
  * the ghost cells a rank's DistributedAdjacencyList adds around its owned
    cells, and the local mesh the kernels then see (``LocalMesh``): owned
    cells first, then ghosts; every face that touches an owned cell, in
    ascending global face id, so each owned cell meets its faces in the
    global order and its sums have the single-rank rounding;
  * ExchangePatternTwoSidedNonBlocking (src/comm/implementation/component/
    ExchangePatternTwoSidedNonBlocking.cpp:129-210): per-peer send lists of
    owned cells and receive ranges of ghost cells (``Halo``); packing and
    unpacking run as kernels of the CUDA library (cupcfd_gpu_dev_halo_pack /
    _unpack), the transfer is NCCL send / recv through torch.distributed
    (``Halo.transfer``).

Local meshes are dicts in the oracle's format (nCells, nFaces, nBnd,
faceCell1/2, faceBnd, geometry, regions) plus the global ids of their cells,
faces and boundaries; a device mesh is made from one with
``Mesh.from_arrays``. Cells owned by the rank come first, so owned outputs
are the first ``nOwned`` cells in local numbering.
"""
from __future__ import annotations

import numpy as np

import cupcfd_b200 as cg


# ---------------------------------------------------------------------------
# partitioning
# ---------------------------------------------------------------------------
def partition_naive(n_cells: int, nparts: int) -> np.ndarray:
    """Part of each cell (label order) as PartitionerNaive assigns it on one
    rank (PartitionerNaive.cpp:97-128): size = n // nparts, remainder
    r = n % nparts; cell i goes to i // size, moved one part down when it
    lies below part*size + min(part, r). (The single step down means that
    with a large remainder the last cells land past the last part; the
    reference's partitioner does the same, and here that raises ValueError.)"""
    if nparts <= 0:
        raise ValueError("nparts must be positive")
    size, rem = n_cells // nparts, n_cells % nparts
    if size == 0:
        raise ValueError("more parts than cells")
    ids = np.arange(n_cells, dtype=np.int64)
    group = ids // size
    check = np.minimum(group, rem)
    down = (group > 0) & (ids < group * size + check)
    part = (group - down).astype(np.int32)
    if part.max() >= nparts:
        raise ValueError(f"the naive assignment puts cells past part {nparts - 1} for {n_cells} cells in "
                         f"{nparts} parts (remainder {rem} against part size {size}); use partition_blocks")
    return part


def partition_blocks(order: np.ndarray, nparts: int) -> np.ndarray:
    """Balanced contiguous blocks of a cell ordering (e.g. a device mesh's
    internal Morton or RCM order from ``Mesh.numbering()``): part of each
    cell label."""
    n = len(order)
    part = np.empty(n, np.int32)
    bounds = np.linspace(0, n, nparts + 1).round().astype(np.int64)
    for p in range(nparts):
        part[order[bounds[p]:bounds[p + 1]]] = p
    return part


# ---------------------------------------------------------------------------
# local meshes
# ---------------------------------------------------------------------------
_FACE_ARRAYS = ("faceLambda", "faceArea", "faceNorm", "faceCenter", "faceXpac", "faceXnac")


class LocalMesh(dict):
    """One rank's part of a mesh (see the module docstring). Extra keys:
    rank, nOwned, cells / faces / bnds (global ids of the local cells, faces
    and boundaries), ghostPart (owner rank of each ghost), send (peer ->
    local ids of the owned cells that peer needs, in the peer's ghost order)
    and recv (peer -> (first, last + 1) local ghost range)."""


def local_mesh(m: dict, part: np.ndarray, rank: int) -> LocalMesh:
    part = np.asarray(part)
    c1 = np.asarray(m["faceCell1"], np.int64)
    c2 = np.asarray(m["faceCell2"], np.int64)
    own = part == rank
    owned = np.flatnonzero(own)
    touch = own[c1] | ((c2 >= 0) & own[np.maximum(c2, 0)])
    faces = np.flatnonzero(touch)
    cells_of_faces = np.concatenate([c1[faces], c2[faces][c2[faces] >= 0]])
    ghosts = np.unique(cells_of_faces[~own[cells_of_faces]])
    ghosts = ghosts[np.lexsort((ghosts, part[ghosts]))]          # by (owner rank, global id)
    cells = np.concatenate([owned, ghosts])
    g2l = -np.ones(int(m["nCells"]), np.int64)
    g2l[cells] = np.arange(len(cells))
    fb = np.asarray(m["faceBnd"], np.int64)[faces]
    bnds = np.sort(fb[fb >= 0])
    b2l = {int(b): i for i, b in enumerate(bnds)}
    out = LocalMesh()
    out["nCells"], out["nFaces"], out["nBnd"] = len(cells), len(faces), len(bnds)
    out["faceCell1"] = g2l[c1[faces]].astype(np.int32)
    out["faceCell2"] = np.where(c2[faces] >= 0, g2l[np.maximum(c2[faces], 0)], -1).astype(np.int32)
    out["faceBnd"] = np.array([b2l[int(b)] if b >= 0 else -1 for b in fb], np.int32)
    for k in _FACE_ARRAYS:
        if m.get(k) is not None:
            out[k] = np.ascontiguousarray(np.asarray(m[k])[faces])
    out["cellCenter"] = np.ascontiguousarray(np.asarray(m["cellCenter"])[cells])
    out["cellVolume"] = np.ascontiguousarray(np.asarray(m["cellVolume"])[cells])
    out["nRegions"] = int(m.get("nRegions", 1))
    for k in ("regionType", "regionUVW", "regionDen"):
        if k in m:
            out[k] = np.asarray(m[k])
    if "bndRegion" in m:
        out["bndRegion"] = np.ascontiguousarray(np.asarray(m["bndRegion"])[bnds]).astype(np.int32)
    out.update(rank=rank, nOwned=len(owned), cells=cells, faces=faces, bnds=bnds, ghostPart=part[ghosts])
    # receive ranges: ghosts are grouped by owner rank
    recv = {}
    for p in np.unique(part[ghosts]):
        idx = np.flatnonzero(part[ghosts] == p) + len(owned)
        recv[int(p)] = (int(idx[0]), int(idx[-1]) + 1)
    out["recv"] = recv
    # send lists: my owned cells that are ghosts of peer p, in p's ghost order
    # (ascending global id); found from the faces between my cells and p's
    send = {}
    cross = (c2 >= 0) & (own[c1] != own[np.maximum(c2, 0)])
    for p in np.unique(part[np.concatenate([c1[cross], c2[cross]])]):
        if p == rank:
            continue
        pm = part == p
        a, b = c1[cross], c2[cross]
        mine = np.concatenate([a[own[a] & pm[b]], b[own[b] & pm[a]]])
        send[int(p)] = g2l[np.unique(mine)].astype(np.int32)
    out["send"] = send
    return out


# ---------------------------------------------------------------------------
# halo exchange on a device mesh
# ---------------------------------------------------------------------------
def exchange_plan(local: LocalMesh):
    """(peers, send, recv, s_off, r_off): the peers in ascending order, the
    concatenated local ids of the cells sent to them and of the ghost cells
    received from them, and each peer's offsets into those lists (the CSR
    sXAdj / rXAdj of the reference's exchange pattern)."""
    peers = sorted(set(local["send"]) | set(local["recv"]))
    send, recv, s_off, r_off = [], [], [0], [0]
    for p in peers:
        sp = local["send"].get(p, np.zeros(0, np.int32))
        lo, hi = local["recv"].get(p, (0, 0))
        send.append(sp)
        recv.append(np.arange(lo, hi))
        s_off.append(s_off[-1] + len(sp))
        r_off.append(r_off[-1] + hi - lo)
    cat = lambda xs: np.concatenate(xs).astype(np.int32) if xs else np.zeros(0, np.int32)
    return peers, cat(send), cat(recv), s_off, r_off


class Halo:
    """The exchange pattern of one local mesh, bound to its device mesh:
    per-peer send and receive index lists in the mesh's internal numbering
    (device int32), in ascending peer order on both sides."""

    def __init__(self, local: LocalMesh, mesh, device):
        import torch
        n2o, _ = mesh.numbering()                       # internal -> local
        o2n = np.empty_like(n2o)
        o2n[n2o] = np.arange(len(n2o), dtype=n2o.dtype)
        self.peers, send, recv, self.s_off, self.r_off = exchange_plan(local)
        self.send_idx = torch.from_numpy(o2n[send].astype(np.int32)).to(device)
        self.recv_idx = torch.from_numpy(o2n[recv].astype(np.int32)).to(device)
        self.device = device

    def buffers(self, ncomp, dtype):
        import torch
        return (torch.empty(max(self.s_off[-1], 1) * ncomp, dtype=dtype, device=self.device),
                torch.empty(max(self.r_off[-1], 1) * ncomp, dtype=dtype, device=self.device))

    @staticmethod
    def _elem(field, ncomp):
        es = field.element_size()
        if field.dim() == 2 and field.shape[1] == 4 and ncomp == 1:   # float4 records as one element
            es *= 4
        return es

    def pack(self, field, sendbuf, ncomp=1, ld=0, stream=None):
        """sendbuf[i * ncomp + c] = field[c * ld + send_idx[i]] (ld defaults
        to the length of one component)."""
        es = self._elem(field, ncomp)
        ld = ld or (field.shape[-1] if ncomp > 1 else 0)
        cg.check(cg.lib().cupcfd_gpu_dev_halo_pack(cg._p(field), es, ncomp, int(ld), cg._p(self.send_idx),
                                                   int(self.s_off[-1]), cg._p(sendbuf), cg._stream(stream)))

    def unpack(self, recvbuf, field, ncomp=1, ld=0, stream=None):
        es = self._elem(field, ncomp)
        ld = ld or (field.shape[-1] if ncomp > 1 else 0)
        cg.check(cg.lib().cupcfd_gpu_dev_halo_unpack(cg._p(recvbuf), es, ncomp, int(self.r_off[-1]),
                                                     cg._p(self.recv_idx), cg._p(field), int(ld), cg._stream(stream)))

    def _fields(self, fields, bufs):
        """HaloField records of [(field, ncomp, ld)] with their buffers."""
        arr = (cg.HaloField * len(fields))()
        for k, ((field, ncomp, ld), buf) in enumerate(zip(fields, bufs)):
            ld = ld or (field.shape[-1] if ncomp > 1 else 0)
            arr[k] = cg.HaloField(field.data_ptr(), self._elem(field, ncomp), ncomp, int(ld), buf.data_ptr())
        return arr

    def pack_fields(self, fields, sendbufs, stream=None):
        """pack() of several fields [(field, ncomp, ld)] in one launch."""
        arr = self._fields(fields, sendbufs)
        cg.check(cg.lib().cupcfd_gpu_dev_halo_pack_fields(arr, len(fields), cg._p(self.send_idx), int(self.s_off[-1]),
                                                          cg._stream(stream)))

    def unpack_fields(self, recvbufs, fields, stream=None):
        """unpack() of several fields [(field, ncomp, ld)] in one launch."""
        arr = self._fields(fields, recvbufs)
        cg.check(cg.lib().cupcfd_gpu_dev_halo_unpack_fields(arr, len(fields), cg._p(self.recv_idx),
                                                            int(self.r_off[-1]), cg._stream(stream)))

    def transfer(self, sendbuf, recvbuf, ncomp=1, words=1, group=None):
        """Each peer's part of sendbuf to that peer, each peer's part of
        recvbuf from it (NCCL for CUDA tensors, gloo for CPU ones). ``words``
        is the number of buffer entries per element and component (4 for a
        float4 record held in a float buffer)."""
        return transfer(self.peers, self.s_off, self.r_off, sendbuf, recvbuf, ncomp * words, group)

    def exchange(self, field, ncomp=1, ld=0, group=None, stream=None):
        """Ghost cells of ``field`` (internal numbering) receive the owners'
        values: pack, transfer, unpack."""
        words = 4 if (field.dim() == 2 and field.shape[1] == 4 and ncomp == 1) else 1
        sendbuf, recvbuf = self.buffers(ncomp * words, field.dtype)
        self.pack(field, sendbuf, ncomp, ld, stream)
        self.transfer(sendbuf, recvbuf, ncomp, words, group)
        self.unpack(recvbuf, field, ncomp, ld, stream)


def transfer(peers, s_off, r_off, sendbuf, recvbuf, per_elem, group=None):
    """The two-sided exchange (ExchangePatternTwoSidedNonBlocking::
    exchangeStart / exchangeStop, :172-210) with torch.distributed: one
    isend and one irecv per peer, batched, then waited on."""
    import torch.distributed as dist
    ops = []
    for i, p in enumerate(peers):
        if r_off[i + 1] > r_off[i]:
            ops.append(dist.P2POp(dist.irecv, recvbuf[r_off[i] * per_elem: r_off[i + 1] * per_elem], p, group))
        if s_off[i + 1] > s_off[i]:
            ops.append(dist.P2POp(dist.isend, sendbuf[s_off[i] * per_elem: s_off[i + 1] * per_elem], p, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
