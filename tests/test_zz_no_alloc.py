"""The remesh entry point for callers that cannot allocate device memory
(pf_remesh_window_noalloc: fixed library-owned scratch, no pf_ctx, no
cudaMalloc/cudaFree).  Such callers are processes whose HBM is already handed
to their own allocator, or threads that must not trigger the device-wide
synchronisation of cudaMalloc/cudaFree.  Checked through the C ABI against the
allocating pf_remesh on two calls in a row, with the device's free memory and
every library context's arena unchanged across the calls.  This file is
collected last on purpose (a failure here leaves every other test run)."""
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


def arenas():
    """Arena bytes of every library context of this process."""
    import pfblob._lib as lb
    out = {}
    for key, h in list(lb._ctx.items()):
        n = ctypes.c_size_t()
        lb.check(lb.lib.pf_mem_usage(h, ctypes.byref(n)))
        out[key] = n.value
    return out


def outputs(capacity):
    xo = torch.full((capacity,), -7.0, dtype=torch.float64, device=DEV)
    return (xo, xo.clone(), xo.clone(), torch.full((capacity,), -7, dtype=torch.int64, device=DEV),
            torch.full((capacity,), -7, dtype=torch.int64, device=DEV),
            torch.zeros(1, dtype=torch.int64, device=DEV),
            torch.full((1,), -1, dtype=torch.int32, device=DEV))


def call(x, y, g, h, xb0, yb0, win, outs):
    import pfblob._lib as lb
    from pfblob._arrays import ptr
    xo, yo, go, ixo, iyo, nout, stat = outs
    st = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    lb.check(lb.lib.pf_remesh_window_noalloc(x.numel(), ptr(x), ptr(y), ptr(g), h, xb0, yb0, 0.0,
                                             *win, xo.numel(), ptr(xo), ptr(yo), ptr(go),
                                             ptr(ixo), ptr(iyo), ptr(nout), ptr(stat), st))


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
    outs = [outputs(cap) for _ in range(2)]
    call(x, y, g, b.h, xb[0], yb[0], win, outputs(cap))  # first call: per-device set-up
    gc.collect()
    torch.cuda.synchronize(DEV)
    free0, _ = torch.cuda.mem_get_info(DEV)
    ar0 = arenas()
    for o in outs:  # two calls in a row share (and must clear) the buffer
        call(x, y, g, b.h, xb[0], yb[0], win, o)
    torch.cuda.synchronize(DEV)
    free1, _ = torch.cuda.mem_get_info(DEV)
    assert free1 == free0, "device memory changed across the calls"
    assert arenas() == ar0, "a library context grew its arena"
    for xo, yo, go, ixo, iyo, nout, stat in outs:
        k = int(nout.item())
        assert int(stat.item()) == 0
        assert k == ref[0].numel()
        for got, want in ((xo, ref[0]), (yo, ref[1]), (ixo, ref[3]), (iyo, ref[4])):
            assert torch.equal(got[:k], want)
        assert (go[:k] - ref[2]).abs().max().item() <= GTOL * ref[2].abs().max().item()
        assert torch.equal(xo[k:], torch.full_like(xo[k:], -7.0))  # nothing beyond the count


def test_noalloc_capacity_overflow_writes_nothing():
    """An output count above the capacity is reported on the device and no
    output entry is written."""
    from pfblob import workloads as wl
    b = wl.lamb_oseen_lattice()
    xb, yb = b.bounds()
    x, y, g = T(b.x), T(b.y), T(b.g)
    win = window(b.x, b.y, b.h, xb[0], yb[0])
    o = outputs(100)
    call(x, y, g, b.h, xb[0], yb[0], win, o)
    torch.cuda.synchronize(DEV)
    assert int(o[5].item()) > 100 and int(o[6].item()) == 0
    assert torch.equal(o[0], torch.full_like(o[0], -7.0))
    assert torch.equal(o[3], torch.full_like(o[3], -7))


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
