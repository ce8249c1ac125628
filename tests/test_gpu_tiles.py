"""The L2-prefetch tile kernels against the plain ones.

Every variant runs the same per-cell arithmetic in the same face order, so
results must be bit-identical:
  - the L2-prefetch kernels (the default when the user arrays start on
    16-byte boundaries) against the plain kernels, which the same call runs
    when phi, gface and the gradient are passed as views offset by one float;
  - the two-launch forward+adjoint (forward with the mass-flux adjoint, then
    the gradient adjoint) against dev_forward + dev_adjoint.
The device timers name the kernels each call ran, so every test checks that
the variant it means to test is the one that ran.

Cases: the Morton, owner and RCM numberings (the native one keeps the
reference's face order, which is not by owner, and has no tile ranges), a
ragged last tile, an odd cell count (the adjoint's gradient blocks are then
not 16-byte aligned, so only the forward takes the tile path), a jittered
mesh.
"""
import os

import pytest

pytestmark = pytest.mark.gpu


def _fields(torch, mesh, seed):
    dev = torch.device("cuda:0")
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
    phi = (torch.rand(nC, generator=g, device=dev, dtype=torch.float64) * 2 - 1).float()
    phiB = (torch.rand(max(nB, 1), generator=g, device=dev, dtype=torch.float64) * 2 - 1).float()
    st = torch.randn(nC, 4, generator=g, device=dev, dtype=torch.float64).float()
    st[:, 0] = 0.9 + 0.2 * torch.rand(nC, generator=g, device=dev, dtype=torch.float64).float()
    gface = torch.randn(nF, generator=g, device=dev, dtype=torch.float64).float()
    return phi, phiB, st.contiguous(), gface


def _offset_copy(torch, t):
    """Same values in a buffer that starts 4 bytes past a 16-byte boundary."""
    buf = torch.empty(t.numel() + 4, dtype=t.dtype, device=t.device)
    v = buf[1:1 + t.numel()].view(t.shape)
    v.copy_(t)
    assert v.data_ptr() % 16 == 4
    return v


def _run(cg, torch, mesh, phi, phiB, st, gface, offset):
    dev = torch.device("cuda:0")
    nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
    if offset:
        phi, gface = _offset_copy(torch, phi), _offset_copy(torch, gface)
        grad = _offset_copy(torch, torch.full((3, nC), float("nan"), device=dev))
    else:
        grad = torch.full((3, nC), float("nan"), device=dev)
    mf = torch.full((nF,), -7.0, device=dev)
    loss = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    pb = torch.full((nC,), float("nan"), device=dev)
    pbb = torch.full((max(nB, 1),), float("nan"), device=dev)
    sb = torch.full((nC, 4), float("nan"), device=dev)
    s = torch.cuda.current_stream()
    cg.timing_read()
    cg.timing_enable(True)
    try:
        cg.dev_forward(mesh, cg.PREC_F32C, phi, phiB, st, grad, mf, gface=gface, loss=loss, stream=s)
        cg.dev_adjoint(mesh, cg.PREC_F32C, grad, st, gface, pb, pbb, sb, stream=s)
        ran = set(cg.timing_read())
    finally:
        cg.timing_enable(False)
    mesh.check_status()
    torch.cuda.synchronize()
    _run.kernels = ran
    return [grad.clone(), mf, loss, pb, pbb, sb]


def _assert_same(a, b):
    import torch
    names = ["grad", "massFlux", "loss", "phiBar", "phiBBar", "stateBar"]
    for n, x, y in zip(names, a, b):
        assert torch.equal(x, y), n
        assert torch.isfinite(x).all(), n


CASES = [
    ("structgen", (12, 10, 8), "ORDER_OWNER"),     # 960 cells: ragged last tile
    ("structgen", (33, 17, 9), "ORDER_MORTON"),    # 5049 cells: odd count
    ("structgen", (40, 32, 24), "ORDER_RCM"),
    ("structgen", (64, 64, 64), "ORDER_OWNER"),    # whole tiles only
    ("jittered", (20, 18, 16), "ORDER_OWNER"),
]


def _mesh(cg, kind, dims, order):
    make = cg.Mesh.structgen if kind == "structgen" else cg.Mesh.jittered
    return make(*dims, order=getattr(cg, order))


@pytest.mark.parametrize("kind,dims,order", CASES)
def test_prefetch_equals_plain(cg, gpu, kind, dims, order):
    import torch
    mesh = _mesh(cg, kind, dims, order)
    fields = _fields(torch, mesh, 5)
    a = _run(cg, torch, mesh, *fields, offset=False)
    ka = _run.kernels
    b = _run(cg, torch, mesh, *fields, offset=True)
    assert "k_fwd_f32_pf" in ka and "k_fwd_f32" in _run.kernels
    if mesh.nCells % 4 == 0:
        assert "k_adj_f32_pf" in ka
    _assert_same(a, b)


def test_native_numbering_runs_plain_kernels(cg, gpu):
    """ORDER_NATIVE keeps the reference's face numbering, which is not sorted
    by owner, so there are no tile ranges and the mesh runs the plain
    kernels."""
    import torch
    mesh = cg.Mesh.structgen(16, 12, 8, order=cg.ORDER_NATIVE)
    assert not mesh.tiles
    _run(cg, torch, mesh, *_fields(torch, mesh, 1), offset=False)
    assert _run.kernels == {"k_fwd_f32", "k_reduce_partials", "k_adj_f32"}


def test_tile_path_can_be_disabled(cg, gpu, monkeypatch):
    import torch
    monkeypatch.setenv("CUPCFD_TILE_MODE", "0")
    off = cg.Mesh.structgen(16, 16, 16, order=cg.ORDER_OWNER)
    monkeypatch.delenv("CUPCFD_TILE_MODE")
    on = cg.Mesh.structgen(16, 16, 16, order=cg.ORDER_OWNER)
    assert not off.tiles and on.tiles
    fields = _fields(torch, on, 3)
    a = _run(cg, torch, off, *fields, offset=False)
    assert _run.kernels == {"k_fwd_f32", "k_reduce_partials", "k_adj_f32"}
    _assert_same(a, _run(cg, torch, on, *fields, offset=False))
    assert "k_fwd_f32_pf" in _run.kernels


def test_misaligned_state_is_rejected(cg, gpu):
    """float4 state records must start on 16-byte boundaries; a misaligned
    pointer is refused before anything is launched."""
    import torch
    mesh = cg.Mesh.structgen(8, 8, 8, order=cg.ORDER_OWNER)
    phi, phiB, st, gface = _fields(torch, mesh, 1)
    bad = _offset_copy(torch, st)
    grad = torch.zeros(3, mesh.nCells, device="cuda:0")
    mf = torch.zeros(mesh.nFaces, device="cuda:0")
    before = cg.launch_count()
    rc = cg.lib().cupcfd_gpu_dev_forward(mesh.h, cg.PREC_F32C, cg._p(phi), cg._p(phiB), cg._p(bad), None,
                                         cg._p(grad), cg._p(mf), None, None)
    assert rc == cg.E_CONFIG_INVALID_VALUE
    assert "16-byte" in cg.last_error()
    assert cg.launch_count() == before


def _run_pipeline(cg, torch, mesh, phi, phiB, st, gface, offset):
    """dev_forward_adjoint; offset views of phi/gface/grad force the plain kernels."""
    dev = torch.device("cuda:0")
    nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
    if offset:
        phi, gface = _offset_copy(torch, phi), _offset_copy(torch, gface)
        grad = _offset_copy(torch, torch.full((3, nC), float("nan"), device=dev))
    else:
        grad = torch.full((3, nC), float("nan"), device=dev)
    mf = torch.full((nF,), -7.0, device=dev)
    loss = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    pb = torch.full((nC,), float("nan"), device=dev)
    pbb = torch.full((max(nB, 1),), float("nan"), device=dev)
    sb = torch.full((nC, 4), float("nan"), device=dev)
    s = torch.cuda.current_stream()
    cg.dev_forward_adjoint(mesh, cg.PREC_F32C, phi, phiB, st, gface, grad, mf, pb, pbb, sb, loss, stream=s)
    mesh.check_status()
    torch.cuda.synchronize()
    return [grad.clone(), mf, loss, pb, pbb, sb]


@pytest.mark.parametrize("kind,dims,order", CASES)
def test_forward_adjoint_pipeline_equals_separate_calls(cg, gpu, kind, dims, order):
    """The two-launch forward+adjoint (mass-flux adjoint moved into the
    forward) equals dev_forward followed by dev_adjoint, bit for bit, and
    so does the same call on offset pointers (plain kernels)."""
    import torch
    make = cg.Mesh.structgen if kind == "structgen" else cg.Mesh.jittered
    mesh = make(*dims, order=getattr(cg, order))
    fields = _fields(torch, mesh, 7)
    ref = _run(cg, torch, mesh, *fields, offset=False)
    _assert_same(_run_pipeline(cg, torch, mesh, *fields, offset=False), ref)
    _assert_same(_run_pipeline(cg, torch, mesh, *fields, offset=True), ref)


@pytest.mark.parametrize("kind,dims,order", [("structgen", (40, 32, 24), "ORDER_RCM"),
                                             ("structgen", (33, 17, 9), "ORDER_MORTON"),
                                             ("jittered", (20, 18, 16), "ORDER_OWNER")])
def test_six_incidence_kernels_equal_general_kernels(cg, gpu, kind, dims, order, monkeypatch):
    """On hexahedral meshes the L2-prefetch kernels run a specialisation for
    cells of exactly six incidences (compile-time trip count, no padding
    checks): the same arithmetic in the same order, so the forward+adjoint
    pipeline, the separate FP32 calls and the FP64 forward give the same bits
    as the general kernels (CUPCFD_FULL_WIDTH=0 at mesh creation)."""
    import torch
    monkeypatch.setenv("CUPCFD_FULL_WIDTH", "0")
    general = _mesh(cg, kind, dims, order)
    monkeypatch.delenv("CUPCFD_FULL_WIDTH")
    six = _mesh(cg, kind, dims, order)
    assert six.tiles and general.tiles and six.full_width == 6 and general.full_width == 0
    fields = _fields(torch, six, 13)
    _assert_same(_run_pipeline(cg, torch, six, *fields, offset=False),
                 _run_pipeline(cg, torch, general, *fields, offset=False))
    _assert_same(_run(cg, torch, six, *fields, offset=False), _run(cg, torch, general, *fields, offset=False))
    phi = fields[0].double()
    phiB = fields[1].double()
    st = fields[2].double().t().contiguous()
    gface = fields[3].double()
    outs = []
    for mesh in (six, general):
        grad = torch.full((3, mesh.nCells), float("nan"), dtype=torch.float64, device="cuda:0")
        mf = torch.zeros(mesh.nFaces, dtype=torch.float64, device="cuda:0")
        loss = torch.zeros(1, dtype=torch.float64, device="cuda:0")
        cg.dev_forward(mesh, cg.PREC_F64, phi, phiB, st, grad, mf, gface=gface, loss=loss,
                       stream=torch.cuda.current_stream())
        mesh.check_status()
        torch.cuda.synchronize()
        outs.append((grad, mf, loss))
    for x, y in zip(*outs):
        assert torch.equal(x, y)


def test_polyhedral_mesh_runs_general_kernels(cg, gpu):
    """Cells of other face counts keep the general kernels."""
    import oracle as O
    m = O.merge_cells(O.jitter(9, 8, 7, 0.25, seed=5, permute=True), 0.4, 11, max_cells=6)
    mesh = cg.Mesh.from_arrays(m, order=cg.ORDER_OWNER)
    assert mesh.tiles and mesh.full_width == 0


def test_device_timers_name_the_pipeline_kernels(cg, gpu):
    """cupcfd_gpu_timing_*: the forward+adjoint call's three launches, each
    timed on its stream, counted per kernel, and cleared by the read."""
    import torch
    mesh = cg.Mesh.structgen(32, 32, 32, order=cg.ORDER_OWNER)
    fields = _fields(torch, mesh, 2)
    cg.timing_read()
    cg.timing_enable(True)
    try:
        for _ in range(3):
            _run_pipeline(cg, torch, mesh, *fields, offset=False)
        t = cg.timing_read()
    finally:
        cg.timing_enable(False)
    assert {k: v[0] for k, v in t.items()} == {"k_fwd_madj_f32_pf": 3, "k_reduce_partials": 3, "k_gadj_f32_pf": 3}
    assert all(v[1] > 0 for v in t.values())
    assert cg.timing_read() == {}


def test_fp64_forward_prefetch_equals_plain(cg, gpu):
    """The FP64 forward and adjoint with the L2 prefetch (16-byte-aligned
    arrays) and the plain ones (phi and the gradient offset by one double)
    give bit-identical results."""
    import torch
    mesh = cg.Mesh.structgen(24, 20, 18, order=cg.ORDER_OWNER)
    dev = torch.device("cuda:0")
    g = torch.Generator(device=dev)
    g.manual_seed(4)
    nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
    phi = torch.rand(nC, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    phiB = torch.rand(nB, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    st = torch.randn(4, nC, generator=g, device=dev, dtype=torch.float64)
    gface = torch.randn(nF, generator=g, device=dev, dtype=torch.float64)
    buf = torch.empty(nC + 2, dtype=torch.float64, device=dev)
    phi_off = buf[1:1 + nC]
    phi_off.copy_(phi)
    assert phi_off.data_ptr() % 16 == 8
    gbuf = torch.empty(3 * nC + 2, dtype=torch.float64, device=dev)
    out = []
    for p, gr in ((phi, torch.empty(3, nC, dtype=torch.float64, device=dev)), (phi_off, gbuf[1:1 + 3 * nC].view(3, nC))):
        gr.fill_(float("nan"))
        mf = torch.zeros(nF, dtype=torch.float64, device=dev)
        loss = torch.zeros(1, dtype=torch.float64, device=dev)
        pb = torch.empty(nC, dtype=torch.float64, device=dev)
        pbb = torch.empty(nB, dtype=torch.float64, device=dev)
        sb = torch.empty(4, nC, dtype=torch.float64, device=dev)
        cg.timing_enable(True)
        try:
            s = torch.cuda.current_stream()
            cg.dev_forward(mesh, cg.PREC_F64, p, phiB, st, gr, mf, gface=gface, loss=loss, stream=s)
            cg.dev_adjoint(mesh, cg.PREC_F64, gr, st, gface, pb, pbb, sb, stream=s)
            names = set(cg.timing_read())
        finally:
            cg.timing_enable(False)
        out.append((gr.clone(), mf, loss, pb, pbb, sb, names))
    assert {"k_fwd_f64_pf", "k_adj_f64_pf"} <= out[0][-1] and {"k_fwd_f64", "k_adj_f64"} <= out[1][-1]
    for a, b in zip(out[0][:-1], out[1][:-1]):
        assert torch.equal(a, b)
