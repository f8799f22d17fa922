"""The coupled blob + panel step (LagrangianSolver.evolve with panels) on the
GPU against the same step restated with the FP64 oracle kernels
(oracle/lagrangian.py, after __lagrangianSolverClass.py:586-677): blob
positions after one coupled RK4 step within 1e-6 (normwise displacement) and
panel strengths within 1e-6, for both panel-strength update modes."""
import numpy as np
import pytest

import oracle
from oracle import lagrangian as olag
from oracle import ref

pytestmark = pytest.mark.gpu


def cylinder(m=96, r=0.5):
    t = np.linspace(0.0, 2.0 * np.pi, m + 1)
    t[-1] = 0.0  # closed contour: last point repeats the first
    return {"cyl": {"xPanel": r * np.cos(t), "yPanel": r * np.sin(t),
                    "cmGlobal": np.array([0.0, 0.0]), "thetaLocal": 0.0, "dPanel": 0.01}}


def cloud(n=3000, seed=3):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.65, 1.2, n)
    a = rng.uniform(-np.pi, np.pi, n)
    return r * np.cos(a), r * np.sin(a), rng.standard_normal(n) / n


@pytest.mark.parametrize("update", ["constant", "varying"])
@pytest.mark.parametrize("method", ["direct", "fmm"])
def test_coupled_rk4_step_matches_oracle_sequence(update, method):
    import pfblob
    if not ref.available():
        pytest.skip("reference Cython panel kernel (oracle/_ref) not built")
    geo = cylinder()
    x, y, g = cloud()
    h, dt, vinf = 0.016, 0.01, (1.0, 0.0)
    blobs = pfblob.Blobs((x, y, g), vInf=list(vinf), nu=0.0, deltaTc=dt, h=h, overlap=0.8,
                         timeIntegrationParams={'method': 'rk4'},
                         velocityComputationParams={'method': method, 'hardware': 'gpu'},
                         blobControlParams={'stepRedistribution': 0, 'stepPopulationControl': 0,
                                            'gThresholdLocal': 1e-8, 'gThresholdGlobal': 1e-8})
    panels = pfblob.Panels(geo)
    solver = pfblob.LagrangianSolver(blobs, panels, couplingParams={'panelStrengthUpdate': update})
    gd = geo["cyl"]
    geom = olag.panel_geometry(gd["xPanel"], gd["yPanel"], gd["cmGlobal"], gd["thetaLocal"])
    assert np.allclose(panels.xyCPGlobalCat, geom[6], rtol=0, atol=1e-15)
    solver.evolve()
    xr, yr, sr = olag.coupled_rk4_step(x, y, g, h / 0.8, geom, vinf, dt, update=update)
    d = np.sqrt((blobs.x - xr) ** 2 + (blobs.y - yr) ** 2)
    disp = np.sqrt((xr - x) ** 2 + (yr - y) ** 2)
    assert d.max() <= 1e-6 * disp.max()
    assert np.abs(panels.sPanel - sr).max() <= 1e-6 * np.abs(sr).max()
    assert solver.tStep == 1 and abs(solver.t - dt) < 1e-15 and panels.tStep == 1


def test_total_velocity_is_blobs_plus_panels_plus_free_stream():
    import pfblob
    geo = cylinder(64)
    x, y, g = cloud(2000, seed=7)
    blobs = pfblob.Blobs((x, y, g), vInf=[0.5, -0.25], nu=0.0, deltaTc=0.01, h=0.016, overlap=0.8,
                         velocityComputationParams={'method': 'direct', 'hardware': 'gpu'},
                         blobControlParams={'stepRedistribution': 0, 'stepPopulationControl': 0,
                                            'gThresholdLocal': 1e-8, 'gThresholdGlobal': 1e-8})
    panels = pfblob.Panels(geo, problemType='fixed')
    solver = pfblob.LagrangianSolver(blobs, panels)
    rng = np.random.default_rng(1)
    xt, yt = rng.uniform(-1.5, 1.5, 500), rng.uniform(-1.5, 1.5, 500)
    vx, vy = solver.evaluateVelocity(xt, yt)
    bx, by = oracle.velocity_direct(x, y, g, 2 * (0.016 / 0.8) ** 2, xt, yt)
    st, en, L, cs = (olag.panel_geometry(geo["cyl"]["xPanel"], geo["cyl"]["yPanel"],
                                         np.zeros(2), 0.0)[k] for k in range(4))
    px, py = oracle.panel_velocity(panels.sPanel, st[0], st[1], en[0], en[1], cs[0], cs[1], xt, yt)
    rx, ry = bx + px + 0.5, by + py - 0.25
    err = np.sqrt((vx - rx) ** 2 + (vy - ry) ** 2).max() / np.sqrt(rx ** 2 + ry ** 2).max()
    assert err <= 1e-6


def test_moving_body_update_and_solve():
    """A 'moving' body (__panelsClass.py:530-637, 715-823): after updateBody
    (translation + rotation) the collocation points follow the reference's
    geometry, the re-assembled influence matrix matches the reference Cython
    kernel, and solve returns the direct solution of A s = -v.t (the
    reference's 'direct' method; its 'gmres'/'bicgstab' approach the same
    solution to their tolerance)."""
    import pfblob
    if not ref.available():
        pytest.skip("reference Cython panel kernel (oracle/_ref) not built")
    geo = cylinder(96)
    panels = pfblob.Panels(geo, problemType='moving',
                           solverCompParams={'method': 'bicgstab', 'tol': 1e-12, 'assemble': 'all'})
    cm, th = np.array([0.3, -0.2]), 0.7
    panels.updateBody({'cyl': cm}, {'cyl': th})
    gd = geo["cyl"]
    st, en, L, cs, norm, tang, cp = olag.panel_geometry(gd["xPanel"], gd["yPanel"], cm, th)
    assert np.allclose(panels.xyCPGlobalCat, cp, rtol=0, atol=1e-15)
    assert np.allclose(panels.normCat, norm, rtol=0, atol=1e-15)
    assert np.allclose(panels.cmGlobal[0], cm) and panels.thetaLocal == [th]
    A = ref.panel_influence(cp[0], cp[1], st[0], st[1], en[0], en[1], cs[0], cs[1])
    assert np.abs(panels.A - A).max() <= 1e-12 * np.abs(A).max()
    rng = np.random.default_rng(11)
    vx, vy = rng.standard_normal(96), rng.standard_normal(96)
    panels.solve(vx, vy)
    rhs = (-vx) * tang[0] + (-vy) * tang[1]
    s_ref = np.linalg.solve(A, rhs)
    assert np.abs(panels.sPanel - s_ref).max() <= 1e-10 * np.abs(s_ref).max()
    # a second move re-assembles again
    panels.updateBody({'cyl': np.array([0.0, 0.0])}, {'cyl': 0.0})
    geom0 = olag.panel_geometry(gd["xPanel"], gd["yPanel"], np.zeros(2), 0.0)
    assert np.allclose(panels.xyCPGlobalCat, geom0[6], rtol=0, atol=1e-15)


def test_update_body_checks_its_arguments():
    import pfblob
    panels = pfblob.Panels(cylinder(32), problemType='moving',
                           solverCompParams={'method': 'direct', 'tol': 1e-12, 'assemble': 'all'})
    with pytest.raises(TypeError):
        panels.updateBody({'other': np.zeros(2)}, {'cyl': 0.1})
    with pytest.raises(TypeError):
        panels.updateBody({'cyl': np.zeros(2)}, {'cyl': 1})
    with pytest.raises(ValueError):
        panels.updateBody({'cyl': np.zeros(3)}, {'cyl': 0.1})
    with pytest.raises(ValueError):
        pfblob.Panels(cylinder(32), problemType='moving',
                      solverCompParams={'method': 'lu', 'tol': 1e-12, 'assemble': 'all'})
