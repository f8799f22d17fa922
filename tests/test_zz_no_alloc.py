"""The remesh entry point for callers that cannot allocate device memory
(pf_remesh_window_noalloc: fixed library-owned scratch, no pf_ctx, no
cudaMalloc/cudaFree).  Checked through the C ABI against the allocating
pf_remesh on two calls in a row; this file is collected last on purpose."""
import ctypes
import gc

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
GTOL = 1e-12


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def window(x, y, h, xb0, yb0):
    ix = oracle.remesh_left_index(x, xb0, h)
    iy = oracle.remesh_left_index(y, yb0, h)
    return int(ix.min()), int(iy.min()), int(ix.max() - ix.min() + 1), int(iy.max() - iy.min() + 1)


def noalloc(x, y, g, h, xb0, yb0, win, capacity):
    import pfblob._lib as lb
    from pfblob._arrays import ptr
    xo = torch.empty(capacity, dtype=torch.float64, device=DEV)
    yo = torch.empty_like(xo)
    go = torch.empty_like(xo)
    ixo = torch.empty(capacity, dtype=torch.int64, device=DEV)
    iyo = torch.empty_like(ixo)
    nout = torch.zeros(1, dtype=torch.int64, device=DEV)
    stat = torch.full((1,), -1, dtype=torch.int32, device=DEV)
    st = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    gc.collect()
    torch.cuda.synchronize(DEV)
    before = torch.cuda.memory_allocated(DEV)
    lb.check(lb.lib.pf_remesh_window_noalloc(x.numel(), ptr(x), ptr(y), ptr(g), h, xb0, yb0, 0.0,
                                             *win, capacity, ptr(xo), ptr(yo), ptr(go), ptr(ixo),
                                             ptr(iyo), ptr(nout), ptr(stat), st))
    torch.cuda.synchronize(DEV)
    assert torch.cuda.memory_allocated(DEV) <= before  # the call allocated nothing
    k = int(nout.item())
    assert int(stat.item()) == 0
    return xo[:k], yo[:k], go[:k], ixo[:k], iyo[:k]


@pytest.mark.parametrize("case", ["lamb_oseen", "uniform"])
def test_noalloc_matches_allocating_remesh_twice(case):
    import pfblob
    from pfblob import workloads as wl
    b = wl.lamb_oseen_lattice() if case == "lamb_oseen" else wl.uniform_square(
        n=150000, sigma=0.004, config=2, instance=11)
    xb, yb = b.bounds()
    x, y, g = T(b.x), T(b.y), T(b.g)
    ref = pfblob.remesh_device(x, y, g, b.h, xb[0], yb[0], with_indices=True)
    win = window(b.x, b.y, b.h, xb[0], yb[0])
    cap = ref[0].numel() + 64
    for _ in range(2):  # two calls in a row share (and must clear) the buffer
        out = noalloc(x, y, g, b.h, xb[0], yb[0], win, cap)
        assert out[0].numel() == ref[0].numel()
        for k in (0, 1, 3, 4):
            assert torch.equal(out[k], ref[k])
        assert (out[2] - ref[2]).abs().max().item() <= GTOL * ref[2].abs().max().item()


def test_noalloc_rejects_sets_beyond_its_buffer():
    import pfblob._lib as lb
    from pfblob._arrays import ptr
    x = torch.zeros(4, dtype=torch.float64, device=DEV)
    n = torch.zeros(1, dtype=torch.int64, device=DEV)
    s = lb.lib.pf_remesh_window_noalloc(4, ptr(x), ptr(x), ptr(x), 0.01, 0.0, 0.0, 0.0, 0, 0,
                                        20000, 20000, 0, None, None, None, None, None, ptr(n),
                                        None, None)
    assert s == 1
    assert b"fixed buffer holds" in lb.lib.pf_last_error()
