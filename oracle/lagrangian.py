"""The coupled blob + panel RK4 step of pHyFlow's LagrangianSolver, restated
with the FP64 oracle kernels (test infrastructure).

Follows ``src/python/lagrangian/__lagrangianSolverClass.py:586-677`` step by
step, with the panel geometry of ``src/python/panels/__panelsClass.py:1009-1058``
and the panel solve of :715-823 ('prescribed': least squares of the influence
matrix plus one total-circulation row, ``numpy.linalg.lstsq``; 'fixed': scipy
LU).  As in the reference, the blob positions are updated in place after each
stage and the next stage's temporary positions start from them.  The
influence matrix comes from the reference's own Cython kernel
(``oracle/_ref``).
"""
import numpy as np
import scipy.linalg

from .core import panel_velocity, velocity_direct
from . import ref


def panel_geometry(xPanel, yPanel, cmGlobal, thetaLocal):
    """(start (2,M), end (2,M), L (M,), cosSin (2,M), norm, tang, cp) of one
    body, with the reference's numpy operations (__panelsClass.py:1009-1058,
    rotation :1094-1096)."""
    rot = np.array([[np.cos(thetaLocal), -np.sin(thetaLocal)],
                    [np.sin(thetaLocal), np.cos(thetaLocal)]])
    xy = np.dot(rot, np.vstack((xPanel, yPanel))) + np.asarray(cmGlobal).reshape(2, 1)
    start, end = xy[:, :-1], xy[:, 1:]
    Lxy = end - start
    L = np.sqrt(np.sum(Lxy * Lxy, axis=0))
    cs = Lxy / L
    norm = np.vstack((-cs[1], cs[0]))
    tang = np.vstack((cs[0], cs[1]))
    cp = 0.5 * (end + start) - norm * L * 0.1
    return start, end, L, cs, norm, tang, cp


def coupled_rk4_step(x, y, g, sigma, geom, vinf, dt, update="constant", problem="prescribed"):
    """One coupled convection step; returns (x, y, panel strengths)."""
    start, end, L, cs, norm, tang, cp = geom
    A = ref.panel_influence(cp[0], cp[1], start[0], start[1], end[0], end[1], cs[0], cs[1])
    M = L.shape[0]
    if problem == "fixed":
        lu = scipy.linalg.lu_factor(A)
    else:
        B = np.zeros((M + 1, M))
        B[:M] = A
        B[M] = L

    def solve(vx, vy):
        rhs = (-vx) * tang[0] + (-vy) * tang[1]
        if problem == "fixed":
            return scipy.linalg.lu_solve(lu, rhs)
        return np.linalg.lstsq(B, np.hstack((rhs, -np.zeros(1))), rcond=None)[0]

    k2 = 2.0 * sigma * sigma
    x, y = x.copy(), y.copy()
    kx = ky = 0
    s = None
    for stage, b, c in zip((1, 2, 3, 4), (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0),
                           (0.0, 0.5, 0.5, 1.0)):
        xt, yt = x + c * dt * kx, y + c * dt * ky
        if update == "varying" or stage == 1:
            vx, vy = velocity_direct(xt, yt, g, k2, cp[0].copy(), cp[1].copy())
            s = solve(vx + vinf[0], vy + vinf[1])
        vxp, vyp = panel_velocity(s, start[0], start[1], end[0], end[1], cs[0], cs[1], xt, yt)
        vxb, vyb = velocity_direct(xt, yt, g, k2, xt, yt)
        kx = vxb + vxp + vinf[0]
        ky = vyb + vyp + vinf[1]
        x += b * kx * dt
        y += b * ky * dt
    return x, y, s
