"""cupcfd_gpu_dev_forward_noalloc: the forward face loops with the loss
reduction, for callers that cannot allocate device memory when they run it
(a solver holding a fixed, pre-reserved memory budget, or code running
inside another runtime that owns the device allocator). It keeps its loss
partials in a fixed array inside the library rather than in the mesh's
scratch pool, so the call itself allocates nothing.

Checked through the C ABI against cupcfd_gpu_dev_forward on the same inputs,
on two calls in a row with different inputs (the shared array keeps the
previous call's contents, which must not leak into the next result). The
two entry points run the same kernels in the same order, so results must be
bit-identical, the tolerance every other FP64 and FP32 kernel-vs-kernel test
here uses. This file is collected last on purpose; it passes alone or after
the other tests (the array's one-time set-up happens on whichever call comes
first).
"""
import pytest

pytestmark = pytest.mark.gpu


def _fields(torch, mesh, prec, seed):
    dev = torch.device("cuda:0")
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    dt = torch.float64 if prec == 0 else torch.float32
    nC, nF, nB = mesh.nCells, mesh.nFaces, mesh.nBoundaries
    phi = (torch.rand(nC, generator=g, device=dev, dtype=torch.float64) * 2 - 1).to(dt)
    phiB = (torch.rand(nB, generator=g, device=dev, dtype=torch.float64) * 2 - 1).to(dt)
    st = torch.randn(4, nC, generator=g, device=dev, dtype=torch.float64).to(dt)
    if prec == 1:
        st = st.t().contiguous()
    gface = torch.randn(nF, generator=g, device=dev, dtype=torch.float64).to(dt)
    return phi, phiB, st, gface


def _outputs(torch, mesh, dt):
    dev = torch.device("cuda:0")
    return (torch.full((3, mesh.nCells), float("nan"), dtype=dt, device=dev),
            torch.zeros(mesh.nFaces, dtype=dt, device=dev),
            torch.full((1,), float("nan"), dtype=torch.float64, device=dev))


@pytest.mark.parametrize("prec", [0, 1])
def test_noalloc_forward_equals_forward_twice(cg, gpu, prec):
    import torch
    mesh = cg.Mesh.structgen(48, 40, 36, order=cg.ORDER_OWNER)
    s = torch.cuda.current_stream()
    for seed in (11, 12):                                    # two calls in a row, different inputs
        phi, phiB, st, gface = _fields(torch, mesh, prec, seed)
        g0, m0, l0 = _outputs(torch, mesh, phi.dtype)
        cg.dev_forward(mesh, prec, phi, phiB, st, g0, m0, gface=gface, loss=l0, stream=s)
        g1, m1, l1 = _outputs(torch, mesh, phi.dtype)
        rc = cg.dev_forward_noalloc(mesh, prec, phi, phiB, st, g1, m1, gface=gface, loss=l1, stream=s)
        assert rc == cg.E_SUCCESS
        assert torch.cuda.current_device() == 0              # the caller's device is given back
        torch.cuda.synchronize()
        assert torch.equal(g0, g1)
        assert torch.equal(m0, m1)
        assert torch.equal(l0, l1) and torch.isfinite(l1).all()


def test_noalloc_rejects_meshes_beyond_its_limit(cg, gpu):
    import torch
    # 257 x 256 x 256 = 16,842,752 cells: 65,792 tiles of 256 cells, beyond the
    # 65,536 tiles (eight loss partials each, one per warp) the fixed array
    # holds
    mesh = cg.Mesh.structgen(257, 256, 256, order=cg.ORDER_OWNER, precisions=1 << cg.PREC_F32C)
    phi, phiB, st, gface = _fields(torch, mesh, 1, 3)
    g, m, l = _outputs(torch, mesh, torch.float32)
    s = torch.cuda.current_stream()
    assert cg.dev_forward_noalloc(mesh, 1, phi, phiB, st, g, m, gface=gface, loss=l, stream=s) == cg.E_ARRAY_SIZE_MISMATCH
    torch.cuda.synchronize()
    assert torch.isnan(g).all()                              # nothing ran
    # without a loss no partials are needed, so the same mesh is accepted
    assert cg.dev_forward_noalloc(mesh, 1, phi, phiB, st, g, m, stream=s) == cg.E_SUCCESS
    torch.cuda.synchronize()
    g0, m0, _ = _outputs(torch, mesh, torch.float32)
    cg.dev_forward(mesh, 1, phi, phiB, st, g0, m0, stream=s)
    torch.cuda.synchronize()
    assert torch.equal(g, g0) and torch.equal(m, m0)
