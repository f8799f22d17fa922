"""StepGraph (pf_step_graph_*): one resident set's velocity + remesh step
captured once as a CUDA graph.  Every replay gives bitwise the result of the
same pf_blob_step issued kernel by kernel, also after the inputs change in
place; the velocity agrees with the FP64 oracle; a launch adds the graph's
kernel nodes to the library's launch counter."""
import ctypes

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def _eager_step(sg, n_out_cap):
    """pf_blob_step with StepGraph sg's descriptor, into fresh output buffers."""
    import pfblob._lib as L
    dev = sg.device
    f64 = dict(dtype=torch.float64, device=dev)
    vx, vy = torch.empty(sg.n, **f64), torch.empty(sg.n, **f64)
    out = torch.empty((3, n_out_cap), **f64)
    n_out = torch.zeros(1, dtype=torch.int64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    mom = torch.zeros(8, **f64)
    d = L.Step()
    ctypes.pointer(d)[0] = sg._desc
    d.vx, d.vy = vx.data_ptr(), vy.data_ptr()
    d.x_out, d.y_out, d.g_out = out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr()
    d.n_out_dev, d.status_dev, d.moments_dev = n_out.data_ptr(), status.data_ptr(), mom.data_ptr()
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    L.check(L.lib.pf_blob_step(L.context(dev.index), ctypes.byref(d), st))
    torch.cuda.synchronize()
    k = int(n_out.item())
    return vx, vy, out[:, :k], int(status.item()), mom


def _set(n, seed):
    rng = np.random.default_rng(seed)
    x, y = rng.random(n), rng.random(n)
    g = rng.standard_normal(n) / n
    return x, y, g


@pytest.mark.parametrize("n", [20000, 131072])
def test_graph_replay_equals_eager_step(n):
    import pfblob
    dev = torch.device("cuda", 0)
    sigma = 0.004
    ks, xopt, cut = pfblob.fmm_parameters(sigma, 2.0, tol=1e-6)
    h = 0.8 * sigma
    x, y, g = (torch.from_numpy(a).to(dev) for a in _set(n, 11))
    box = (0.0, 1.0, 0.0, 1.0)
    sg = pfblob.StepGraph(x, y, g, ks, xopt, cut, 1e-6, box, h, -1.5 * h, -1.5 * h,
                          max_base_cells=4 * int((1.0 / h + 8) ** 2))
    assert sg.kernels >= 20
    for it in range(2):
        if it:  # new values in the same buffers (a stepping loop moves its blobs)
            rng = np.random.default_rng(5)
            x.add_(torch.from_numpy(rng.uniform(-1e-3, 1e-3, n)).to(dev)).clamp_(0.0, 1.0)
            g.mul_(1.5)
        from pfblob import _lib
        l0 = _lib.kernel_launches()
        sg.launch()
        assert _lib.kernel_launches() - l0 == sg.kernels
        xo, yo, go, status = sg.result()
        assert status == 0
        vx, vy, out, st_e, mom = _eager_step(sg, sg.out.shape[1])
        assert st_e == 0
        assert torch.equal(sg.vx, vx) and torch.equal(sg.vy, vy)
        assert out.shape[1] == xo.numel()
        assert torch.equal(out[0], xo) and torch.equal(out[1], yo) and torch.equal(out[2], go)
        assert torch.equal(sg.moments, mom)
    # velocity against the FP64 direct Gauss sum on a target subset
    idx = np.arange(0, n, max(1, n // 512))
    xs, ys, gs = x.cpu().numpy(), y.cpu().numpy(), g.cpu().numpy()
    ux, uy = oracle.velocity_direct(xs, ys, gs, ks, xs[idx], ys[idx])
    gx, gy = sg.vx.cpu().numpy()[idx], sg.vy.cpu().numpy()[idx]
    err = np.sqrt(np.sum((gx - ux) ** 2 + (gy - uy) ** 2) / np.sum(ux ** 2 + uy ** 2))
    assert err < 1e-6, err
    # circulation is conserved by the remesh (FP64 moments before and after)
    m = sg.moments.cpu().numpy()
    assert abs(m[4] - m[0]) <= 1e-12 * max(m[3], 1e-300)
    sg.close()
    sg.close()
    with pytest.raises(ValueError):
        sg.launch()


def test_graph_reports_window_beyond_its_bound():
    """A step whose remesh window exceeds the graph's bound sets status bit 8
    and writes no blob, like pf_remesh_async; the graph stays usable."""
    import pfblob
    dev = torch.device("cuda", 0)
    n = 4096
    sigma = 0.01
    ks, xopt, cut = pfblob.fmm_parameters(sigma, 2.0, tol=1e-6)
    h = 0.8 * sigma
    x, y, g = (torch.from_numpy(a).to(dev) for a in _set(n, 3))
    # tree box [0, 2]^2, remesh bound for blobs in [0, 1]^2
    sg = pfblob.StepGraph(x, y, g, ks, xopt, cut, 1e-6, (0.0, 2.0, 0.0, 2.0), h, -1.5 * h,
                          -1.5 * h, max_base_cells=int((1.0 / h + 8) ** 2))
    sg.launch()
    assert sg.result()[3] == 0
    x.mul_(2.0)  # the blobs now span [0, 2] x [0, 1]: twice the window
    sg.launch()
    assert sg.result()[3] & 8
    x.mul_(0.5)
    sg.launch()
    assert sg.result()[3] == 0
    sg.close()


def test_direct_method_graph_equals_eager_step():
    """The direct-sum step (method = PF_DIRECT_METHOD) captured and replayed:
    bitwise the eager pf_blob_step, and within 1e-6 of the FP64 oracle."""
    import pfblob
    dev = torch.device("cuda", 0)
    n = 6000
    sigma = 0.01
    ks, xopt, cut = pfblob.fmm_parameters(sigma, 2.0, tol=1e-6)
    h = 0.8 * sigma
    x, y, g = (torch.from_numpy(a).to(dev) for a in _set(n, 9))
    sg = pfblob.StepGraph(x, y, g, ks, xopt, cut, 1e-6, (0.0, 1.0, 0.0, 1.0), h, -1.5 * h,
                          -1.5 * h, method=pfblob.DIRECT_METHOD,
                          max_base_cells=4 * int((1.0 / h + 8) ** 2))
    sg.launch()
    xo, yo, go, status = sg.result()
    assert status == 0 and xo.numel() > 0
    vx, vy, out, st_e, mom = _eager_step(sg, sg.out.shape[1])
    assert st_e == 0
    assert torch.equal(sg.vx, vx) and torch.equal(sg.vy, vy)
    assert torch.equal(out[2], go)
    xs, ys, gs = x.cpu().numpy(), y.cpu().numpy(), g.cpu().numpy()
    ux, uy = oracle.velocity_direct(xs, ys, gs, ks)
    gx, gy = sg.vx.cpu().numpy(), sg.vy.cpu().numpy()
    err = np.sqrt(np.sum((gx - ux) ** 2 + (gy - uy) ** 2) / np.sum(ux ** 2 + uy ** 2))
    assert err < 1e-6, err
    sg.close()
