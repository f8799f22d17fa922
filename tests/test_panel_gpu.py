"""Vortex-panel velocity on the GPU vs the reference Cython kernel (golden)
and the oracle.  Gate: normwise relative error <= 1e-6."""
import numpy as np
import pytest
import torch

import oracle
from conftest import normwise_err

pytestmark = pytest.mark.gpu
TOL = 1e-6


def test_cylinder_vs_reference_golden(golden):
    import pfblob
    p = golden("panel_cyl")
    vx, vy = pfblob.inducedVelocity(p["gamma"], p["xs"], p["ys"], p["xe"], p["ye"], p["cosa"],
                                    p["sina"], p["xv"], p["yv"])
    # the point 1e-6 from the panel (index 3) has a large, well-defined value
    assert normwise_err(vx[4:], vy[4:], p["vx"][4:], p["vy"][4:]) <= TOL
    assert abs(vx[3] - p["vx"][3]) <= 1e-5 * abs(p["vx"][3]) + 1e-6
    # on the line extension of a panel: finite and equal to the reference
    assert np.allclose(vx[:3], p["vx"][:3], rtol=1e-5, atol=1e-7)


def test_512_panels_shear_layer_points():
    import pfblob
    from pfblob import workloads as wl
    ps = wl.cylinder_panels(512)
    rng = np.random.default_rng(2)
    r = rng.uniform(1.0, 1.5, 20000)
    t = rng.uniform(-np.pi, np.pi, 20000)
    xv, yv = r * np.cos(t), r * np.sin(t)
    rx, ry = oracle.panel_velocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina, xv, yv)
    vx, vy = pfblob.inducedVelocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina, xv, yv)
    assert normwise_err(vx, vy, rx, ry) <= TOL


def test_accumulate_onto_blob_velocity():
    import pfblob
    from pfblob import workloads as wl
    ps = wl.cylinder_panels(64)
    dev = torch.device("cuda", 0)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    xv = T(np.linspace(-2, 2, 1000))
    yv = T(np.full(1000, 1.7))
    vx = torch.full((1000,), 0.25, dtype=torch.float64, device=dev)
    vy = torch.full((1000,), -0.5, dtype=torch.float64, device=dev)
    pfblob.panel_velocity_device(T(ps.gamma), T(ps.xs), T(ps.ys), T(ps.xe), T(ps.ye), T(ps.cosa),
                                 T(ps.sina), xv, yv, vx, vy, accumulate=True)
    rx, ry = oracle.panel_velocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina,
                                   xv.cpu().numpy(), yv.cpu().numpy())
    assert normwise_err(vx.cpu().numpy() - 0.25, vy.cpu().numpy() + 0.5, rx, ry) <= TOL


def test_far_points_series_to_1e10():
    """Points well away from the body take the groups' series only: they match
    the FP64 pair formula to 1e-10 (the series' stated remainder), far inside
    the 1e-6 gate that the FP32 transcendentals of the near field set."""
    import pfblob
    from pfblob import workloads as wl
    ps = wl.cylinder_panels(512)
    rng = np.random.default_rng(4)
    r = rng.uniform(2.0, 6.0, 20000)
    t = rng.uniform(-np.pi, np.pi, 20000)
    xv, yv = r * np.cos(t), r * np.sin(t)
    rx, ry = oracle.panel_velocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina, xv, yv)
    vx, vy = pfblob.inducedVelocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina, xv, yv)
    assert normwise_err(vx, vy, rx, ry) <= 1e-10


def test_shuffled_panels_and_many_groups():
    """The grouping never changes the sum: panels in random order (every group
    spans the body, so every point is near) and a body of 1000 panels (a
    partial last group, several shared-memory tiles) both meet the gate."""
    import pfblob
    from pfblob import workloads as wl
    rng = np.random.default_rng(6)
    r = rng.uniform(1.0, 3.0, 8000)
    t = rng.uniform(-np.pi, np.pi, 8000)
    xv, yv = r * np.cos(t), r * np.sin(t)
    for m, shuffle in ((512, True), (1000, False), (1000, True)):
        ps = wl.cylinder_panels(m)
        arrs = [ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina]
        if shuffle:
            perm = rng.permutation(m)
            arrs = [a[perm] for a in arrs]
        rx, ry = oracle.panel_velocity(*arrs, xv, yv)
        vx, vy = pfblob.inducedVelocity(*arrs, xv, yv)
        assert normwise_err(vx, vy, rx, ry) <= TOL, (m, shuffle)


def test_source_panels_vs_reference_golden(golden):
    """Constant-source panels (panelKernel=0): velocity against the
    reference's Cython kernel (gate 1e-6; the point 1e-6 from panel 0 and the
    points on its line extension as for vortex panels) and the influence
    matrix against its assemble_influenceMatrix (1e-12)."""
    import pfblob
    d = golden("source_panel")
    args = [d[k] for k in ("sigma", "xs", "ys", "xe", "ye", "cosa", "sina")]
    vx, vy = pfblob.inducedVelocity(*args, d["xv"], d["yv"], panelKernel=0)
    assert normwise_err(vx[4:], vy[4:], d["vx"][4:], d["vy"][4:]) <= TOL
    e3 = np.hypot(vx[3] - d["vx"][3], vy[3] - d["vy"][3])
    assert e3 <= 1e-5 * np.hypot(d["vx"][3], d["vy"][3]) + 1e-6
    assert np.allclose(vx[:3], d["vx"][:3], rtol=1e-5, atol=1e-7)
    assert np.allclose(vy[:3], d["vy"][:3], rtol=1e-5, atol=1e-7)
    A = pfblob.influenceMatrix(d["xcp"], d["ycp"], *args[1:], panelKernel=0)
    assert np.abs(A - d["A"]).max() <= 1e-12 * np.abs(d["A"]).max()


def test_source_panels_far_field_and_panels_class():
    """Far points take the groups' series only (1e-10 against the FP64
    oracle); a 'css' Panels body solves the no-through-flow condition
    (RHS = -v.n) with the source influence matrix."""
    import pfblob
    from pfblob import workloads as wl
    ps = wl.cylinder_panels(512)
    rng = np.random.default_rng(8)
    r = rng.uniform(2.0, 6.0, 8000)
    t = rng.uniform(-np.pi, np.pi, 8000)
    xv, yv = r * np.cos(t), r * np.sin(t)
    args = (ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina)
    rx, ry = oracle.source_panel_velocity(*args, xv, yv)
    vx, vy = pfblob.inducedVelocity(*args, xv, yv, panelKernel=0)
    assert normwise_err(vx, vy, rx, ry) <= 1e-10
    m = 64
    th = np.linspace(0.0, 2.0 * np.pi, m + 1)
    th[-1] = 0.0
    geo = {"b": {"xPanel": 0.5 * np.cos(th), "yPanel": 0.5 * np.sin(th),
                 "cmGlobal": np.array([0.1, 0.2]), "thetaLocal": 0.3, "dPanel": 0.01}}
    panels = pfblob.Panels(geo, panelKernel='css', problemType='fixed')
    vxe, vye = rng.standard_normal(m), rng.standard_normal(m)
    panels.solve(vxe, vye)
    n = panels.normCat
    rhs = (-vxe) * n[0] + (-vye) * n[1]
    s_ref = np.linalg.solve(panels.A, rhs)
    assert np.abs(panels.sPanel - s_ref).max() <= 1e-10 * np.abs(s_ref).max()
    assert np.all(np.asarray(panels.gTotal) == 0.0)


def _annulus(n, r0, r1, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(r0, r1, n)
    t = rng.uniform(-np.pi, np.pi, n)
    return r * np.cos(t), r * np.sin(t)


def test_box_grid_path_near_wall_vs_oracle():
    """2^16 points (the box-grid path: far groups through each box's local
    expansion, near groups per point) in the near-wall annulus: the gate."""
    import pfblob
    from pfblob import workloads as wl
    ps = wl.cylinder_panels(512)
    xv, yv = _annulus(1 << 16, 1.0, 1.5, 8)
    rx, ry = oracle.panel_velocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina, xv, yv)
    vx, vy = pfblob.inducedVelocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina, xv, yv)
    assert normwise_err(vx, vy, rx, ry) <= TOL


def test_box_grid_path_far_points_to_1e10():
    """Far points on the box-grid path carry every group through the local
    expansions: still within 1e-10 of the FP64 pair formula."""
    import pfblob
    from pfblob import workloads as wl
    ps = wl.cylinder_panels(512)
    xv, yv = _annulus(1 << 16, 2.0, 6.0, 9)
    rx, ry = oracle.panel_velocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina, xv, yv)
    vx, vy = pfblob.inducedVelocity(ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina, xv, yv)
    assert normwise_err(vx, vy, rx, ry) <= 1e-10


@pytest.mark.parametrize("m,shuffle", [(512, False), (2048, False), (512, True)])
def test_box_grid_path_as_accurate_as_per_point_path(m, shuffle):
    """The same points through both paths (40,000 at once: box grid; 10,000
    at a time: every group per point) against the FP64 oracle: the box grid
    meets the gate with the per-point path's accuracy (both are set by the
    FP32 transcendentals of the pair formula at the points nearest the body;
    the box grid takes the FP64 series of sub-groups for more of its near
    panels); also with shuffled panels, whose groups span the body."""
    import pfblob
    from pfblob import workloads as wl
    ps = wl.cylinder_panels(m)
    arrs = [ps.gamma, ps.xs, ps.ys, ps.xe, ps.ye, ps.cosa, ps.sina]
    if shuffle:
        perm = np.random.default_rng(10).permutation(m)
        arrs = [a[perm] for a in arrs]
    xv, yv = _annulus(40000, 1.0, 3.0, 11)
    vx, vy = pfblob.inducedVelocity(*arrs, xv, yv)
    px, py = [], []
    for k in range(0, 40000, 10000):
        a, b = pfblob.inducedVelocity(*arrs, xv[k:k + 10000], yv[k:k + 10000])
        px.append(a)
        py.append(b)
    px, py = np.concatenate(px), np.concatenate(py)
    rx, ry = oracle.panel_velocity(*arrs, xv, yv)
    e_box, e_pt = normwise_err(vx, vy, rx, ry), normwise_err(px, py, rx, ry)
    assert e_box <= TOL and e_box <= 1.5 * e_pt + 1e-10, (e_box, e_pt)
