"""A mesh split across ranks, run on one GPU: three local meshes (owned cells,
then ghosts; internal Morton numbering, so the exchange lists are
permuted), the halo pack / unpack kernels of the library, and the transfer
between ranks emulated by device copies of each peer's part of the send
buffer into the receiving rank's buffer (one GPU cannot host NCCL ranks;
the NCCL transfer, halo.transfer, is covered by the two-rank gloo test on
CPU). Forward + adjoint in FP64 and FP32-compensated, with the state
exchanged before the forward and the gradient between forward and adjoint
(as a multi-rank step does), give on every owned cell and owned face the
bits of the single-mesh run.
"""
import numpy as np
import pytest

import oracle as O
from conftest import load_cupcfd

pytestmark = pytest.mark.gpu


def _setup(kind, nparts=3):
    load_cupcfd()
    import cupcfd_b200.halo as H
    if kind == "poly":
        m = O.merge_cells(O.jitter(16, 14, 12, 0.25, seed=6, permute=True), 0.35, 3, max_cells=4)
    else:
        m = O.jitter(18, 16, 14, 0.25, seed=2, permute=True)
    part = H.partition_blocks(np.argsort(m["cellCenter"][:, 2] + 0.1 * m["cellCenter"][:, 0]), nparts)
    return H, m, part


def _emulated_exchange(halos, fields, ncomp=1, ld=0, words=1):
    """pack on every rank, copy each peer's part to it, unpack."""
    import torch
    bufs = [h.buffers(ncomp * words, f.dtype) for h, f in zip(halos, fields)]
    for h, f, (sb, _) in zip(halos, fields, bufs):
        h.pack(f, sb, ncomp, ld)
    k = ncomp * words
    for r, h in enumerate(halos):
        for i, p in enumerate(h.peers):
            hp = halos[p]
            j = hp.peers.index(r)
            src = bufs[r][0][h.s_off[i] * k: h.s_off[i + 1] * k]
            dst = bufs[p][1][hp.r_off[j] * k: hp.r_off[j + 1] * k]
            assert src.numel() == dst.numel()
            dst.copy_(src)
    for h, f, (_, rb) in zip(halos, fields, bufs):
        h.unpack(rb, f, ncomp, ld)
    torch.cuda.synchronize()


@pytest.mark.parametrize("kind", ["jitter", "poly"])
@pytest.mark.parametrize("prec", [0, 1])
def test_sharded_forward_adjoint_equals_single_mesh(cg, gpu, kind, prec):
    import torch
    H, m, part = _setup(kind)
    dev = torch.device("cuda:0")
    dt = torch.float64 if prec == cg.PREC_F64 else torch.float32
    f = O.fields(m, 21)
    gface = np.random.Generator(np.random.Philox(key=22)).standard_normal(m["nFaces"])

    def T(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    def run(mesh, phi_l, phiB_l, state_l, gface_l, exchange_grad=None):
        """forward, optional gradient exchange, adjoint; inputs in the mesh's
        reference (local) numbering, moved to internal with the library."""
        nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
        phi = torch.empty(nC, dtype=dt, device=dev)
        cg.permute_cells(mesh, True, T(phi_l).to(dt), phi)
        st_ref = T(state_l).to(dt)                                  # [4][nC] reference order
        if prec == cg.PREC_F64:
            st = torch.empty(4, nC, dtype=dt, device=dev)
            cg.permute_cells(mesh, True, st_ref, st, ncomp=4)
        else:
            st_b = torch.empty(4, nC, dtype=dt, device=dev)
            cg.permute_cells(mesh, True, st_ref, st_b, ncomp=4)
            st = st_b.t().contiguous()                              # float4 records
        gf = torch.empty(nF, dtype=dt, device=dev)
        cg.permute_faces(mesh, True, T(gface_l).to(dt), gf)
        return dict(phi=phi, phiB=T(phiB_l).to(dt), st=st, gf=gf)

    def forward(mesh, x):
        nC, nF = mesh.nCells, mesh.nFaces
        x["grad"] = torch.empty(3, nC, dtype=dt, device=dev)
        x["mf"] = torch.zeros(nF, dtype=dt, device=dev)
        cg.dev_forward(mesh, prec, x["phi"], x["phiB"], x["st"], x["grad"], x["mf"], stream=torch.cuda.current_stream())

    def adjoint(mesh, x):
        nC, nB = mesh.nCells, mesh.nBoundaries
        x["pb"] = torch.empty(nC, dtype=dt, device=dev)
        x["pbb"] = torch.empty(max(nB, 1), dtype=dt, device=dev)
        x["sb"] = torch.empty_like(x["st"])
        cg.dev_adjoint(mesh, prec, x["grad"], x["st"], x["gf"], x["pb"], x["pbb"], x["sb"],
                       stream=torch.cuda.current_stream())
        torch.cuda.synchronize()

    def to_ref(mesh, x):
        """outputs in the mesh's reference numbering (host FP64)."""
        c2o, f2o = mesh.numbering()
        out = {}
        g = x["grad"].double().cpu().numpy()
        out["grad"] = np.empty((mesh.nCells, 3))
        out["grad"][c2o] = g.T
        for k in ("pb",):
            out[k] = np.empty(mesh.nCells)
            out[k][c2o] = x[k].double().cpu().numpy()
        sb = x["sb"].double().cpu().numpy()
        sb = sb.T if prec == cg.PREC_F64 else sb
        out["sb"] = np.empty((mesh.nCells, 4))
        out["sb"][c2o] = sb
        out["mf"] = np.empty(mesh.nFaces)
        out["mf"][f2o] = x["mf"].double().cpu().numpy()
        out["pbb"] = x["pbb"].double().cpu().numpy()[:mesh.nBoundaries]
        return out

    state = np.stack([f["den"], f["u"], f["v"], f["w"]])
    gm = cg.Mesh.from_arrays(m, order=cg.ORDER_MORTON)
    gx = run(gm, f["phi"], f["phiB"], state, gface)
    forward(gm, gx)
    adjoint(gm, gx)
    want = to_ref(gm, gx)

    locs = [H.local_mesh(m, part, r) for r in range(3)]
    meshes = [cg.Mesh.from_arrays(l, order=cg.ORDER_MORTON) for l in locs]
    halos = [H.Halo(l, me, dev) for l, me in zip(locs, meshes)]
    xs = []
    for l, me in zip(locs, meshes):
        nO = l["nOwned"]
        phi_l = f["phi"][l["cells"]].copy()
        st_l = state[:, l["cells"]].copy()
        phi_l[nO:] = np.nan                                          # ghosts come from the exchange
        st_l[:, nO:] = np.nan
        xs.append(run(me, phi_l, f["phiB"][l["bnds"]], st_l, gface[l["faces"]]))
    _emulated_exchange(halos, [x["phi"] for x in xs])
    if prec == cg.PREC_F64:
        _emulated_exchange(halos, [x["st"] for x in xs], ncomp=4, ld=0)
    else:
        _emulated_exchange(halos, [x["st"] for x in xs], words=4)
    for me, x in zip(meshes, xs):
        forward(me, x)
    _emulated_exchange(halos, [x["grad"] for x in xs], ncomp=3)
    for me, x in zip(meshes, xs):
        adjoint(me, x)
    for l, me, x in zip(locs, meshes, xs):
        got = to_ref(me, x)
        nO, cells = l["nOwned"], l["cells"][:l["nOwned"]]
        for k in ("grad", "pb", "sb"):
            assert np.array_equal(got[k][:nO], want[k][cells]), (l["rank"], k)
        own_f = part[m["faceCell1"][l["faces"]]] == l["rank"]
        inner = m["faceCell2"][l["faces"]] >= 0
        sel = own_f & inner
        assert np.array_equal(got["mf"][sel], want["mf"][l["faces"][sel]]), l["rank"]
        assert np.array_equal(got["pbb"], want["pbb"][l["bnds"]]), l["rank"]


def test_pack_unpack_layouts(cg, gpu):
    """pack / unpack against numpy on the element sizes and layouts used."""
    import torch
    H, m, part = _setup("jitter")
    dev = torch.device("cuda:0")
    l = H.local_mesh(m, part, 1)
    me = cg.Mesh.from_arrays(l, order=cg.ORDER_RCM)
    h = H.Halo(l, me, dev)
    si, ri = h.send_idx.cpu().numpy(), h.recv_idx.cpu().numpy()
    rng = np.random.default_rng(1)
    for dt, shape, ncomp in ((torch.float64, (me.nCells,), 1), (torch.float32, (3, me.nCells), 3),
                             (torch.float64, (4, me.nCells), 4), (torch.float32, (me.nCells, 4), 1)):
        field = torch.from_numpy(rng.standard_normal(shape)).to(dt).to(dev)
        words = 4 if shape == (me.nCells, 4) else 1
        sb, rb = h.buffers(ncomp * words, dt)
        h.pack(field, sb, ncomp)
        fn = field.cpu().numpy()
        if words == 4:
            want = fn[si].reshape(-1)
        else:
            want = (fn.reshape(ncomp, -1)[:, si].T).reshape(-1)
        assert np.array_equal(sb.cpu().numpy()[:len(want)], want)
        src = torch.from_numpy(rng.standard_normal(rb.numel())).to(dt).to(dev)
        h.unpack(src, field, ncomp)
        fn2 = fn.copy()
        s = src.cpu().numpy()[:len(ri) * ncomp * words]
        if words == 4:
            fn2[ri] = s.reshape(-1, 4)
        else:
            fn2.reshape(ncomp, -1)[:, ri] = s.reshape(-1, ncomp).T
        assert np.array_equal(field.cpu().numpy(), fn2)


def test_pack_fields_equals_single_field_calls(cg, gpu):
    """The multi-field pack / unpack (one launch per direction) moves the
    same bits as one single-field call per field: scalar, float4 record and
    three-component fields, FP32 and FP64."""
    import torch
    H, m, part = _setup("jitter")
    dev = torch.device("cuda:0")
    loc = H.local_mesh(m, part, 1)
    mesh = cg.Mesh.from_arrays(loc)
    h = H.Halo(loc, mesh, dev)
    nC = mesh.nCells
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    fields = [(torch.rand(nC, generator=g, device=dev), 1, 0),
              (torch.rand(nC, 4, generator=g, device=dev), 1, 0),
              (torch.rand(3, nC, generator=g, device=dev, dtype=torch.float64), 3, nC)]
    words = [1, 4, 1]
    single = [h.buffers(nc * w, f.dtype)[0] for (f, nc, _), w in zip(fields, words)]
    for (f, nc, ld), b in zip(fields, single):
        h.pack(f, b, nc, ld)
    multi = [torch.full_like(b, float("nan")) for b in single]
    h.pack_fields(fields, multi)
    torch.cuda.synchronize()
    for a, b in zip(single, multi):
        assert torch.equal(a, b)
    # unpack random buffers into copies of the fields both ways
    recv = [torch.rand(max(h.r_off[-1], 1) * nc * w, generator=g, device=dev, dtype=f.dtype)
            for (f, nc, _), w in zip(fields, words)]
    one = [f.clone() for f, _, _ in fields]
    for (f, nc, ld), r, o in zip(fields, recv, one):
        h.unpack(r, o, nc, ld)
    both = [f.clone() for f, _, _ in fields]
    h.unpack_fields(recv, [(o, nc, ld) for o, (_, nc, ld) in zip(both, fields)])
    torch.cuda.synchronize()
    for a, b in zip(one, both):
        assert torch.equal(a, b)
    # more than 8 fields is refused
    arr = (cg.HaloField * 9)()
    assert cg.lib().cupcfd_gpu_dev_halo_pack_fields(arr, 9, cg._p(h.send_idx), 1, None) == cg.E_CONFIG_INVALID_VALUE
