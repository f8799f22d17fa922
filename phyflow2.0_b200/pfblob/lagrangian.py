"""Vortex panels and the coupled blob + panel solver with pHyFlow's call
surface, state on the GPU.

``Panels`` mirrors the parts of ``pHyFlow.panels.Panels``
(``src/python/panels/__panelsClass.py``) that the Lagrangian step uses: the
body geometry (rotation by thetaLocal about cmGlobal, panel ends, normals,
tangents, collocation points moved inside by a tenth of the panel length,
:964-1058), the influence matrix (:872-962, ``pf_panel_influence_matrix``),
``solve`` (:715-823; 'fixed' by LU, 'prescribed' by the least-squares system
of the influence matrix plus one total-circulation row per body, 'moving' by
the direct solve of the re-assembled matrix), ``updateBody`` (:530-637: new
cmGlobal and thetaLocal, coordinates and influence matrix rebuilt) and
``evaluateVelocity`` (:641-712, ``pf_panel_velocity``), for constant-
strength vortex ('csv') or source ('css') panels.  For a moving body the reference
solves with scipy's 'gmres' or 'bicgstab' to its 'tol', or 'direct'
(``numpy.linalg.solve``); every method here is the direct solve by LU on the
GPU, the solution the iterations approach.

``LagrangianSolver`` mirrors ``pHyFlow.lagrangian.LagrangianSolver``
(``src/python/lagrangian/__lagrangianSolverClass.py``): ``evaluateVelocity``
(:202-266, blob + panel + free-stream velocity) and ``evolve`` (:270-368) with
the coupled RK4 convection (:586-677), diffusion, redistribution and
population control.  The reference's coupled RK4 reads the blob positions
through the ``Blobs.x`` property, which returns the array itself, and adds
each stage's increment to that same array: a stage's temporary positions are
the positions already moved by the earlier stages plus c_k dt k_{k-1}.  That
is what the reference computes, and what ``evolve`` computes here.
"""
import numpy as np
import torch

from . import _lib
from ._arrays import ptr
from .induced import DIRECT_METHOD, FMM_METHOD, fmm_parameters, velocity_device
from .panels import PANEL_KERNEL_CSS, PANEL_KERNEL_CSV, panel_velocity_device

PANEL_KERNELS = ('csv', 'css')
PROBLEM_TYPES = ('fixed', 'moving', 'prescribed')
PANEL_STRENGTH_UPDATES = ('constant', 'varying')


def _lu(dev, a):
    """LU factors (row-major, partial pivoting) of a square device matrix."""
    n = a.shape[0]
    lu = a.clone()
    piv = torch.empty(n, dtype=torch.int32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    _lib.check(_lib.lib.pf_dense_lu_factor(_lib.context(dev.index), n, ptr(lu), ptr(piv),
                                           ptr(info), st))
    return lu, piv


def _lu_solve(dev, lu, piv, b):
    x = b.clone()
    st = torch.cuda.current_stream(dev).cuda_stream
    _lib.check(_lib.lib.pf_dense_lu_solve(_lib.context(dev.index), x.numel(), ptr(lu), ptr(piv),
                                          ptr(x), st))
    return x


class Panels:
    """Straight constant-strength vortex panels on fixed bodies, on the GPU."""

    def __init__(self, geometries, panelKernel='csv', problemType='prescribed',
                 velCompParams={'method': 'direct', 'hardware': 'cpu'},
                 solverCompParams={'method': 'bicgstab', 'tol': 1e-12, 'assemble': 'all'},
                 device=None):
        if type(geometries) != dict:
            raise TypeError("'geometries' must either be a dictionary of geometries, containing "
                            "all the parameters of its body: ['xPanel','yPanel','cmGlobal',"
                            "'thetaLocal', 'dPanel'] in a dictionary format.")
        if panelKernel not in PANEL_KERNELS:
            raise ValueError("panelKernel must be one of %s" % str(PANEL_KERNELS))
        if problemType not in PROBLEM_TYPES:
            raise ValueError("problemType must be one of %s" % str(PROBLEM_TYPES))
        if problemType == 'moving' and solverCompParams.get('method') not in (
                'gmres', 'bicgstab', 'direct'):
            raise ValueError("solverCompParams['method'] must be one of "
                             "('gmres', 'bicgstab', 'direct') for a moving problem")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None
                                   else device)
        self._panelKernel = panelKernel
        self._problemType = problemType
        self._velCompParams = dict(velCompParams)
        self._solverCompParams = dict(solverCompParams)
        keys = ['xPanel', 'yPanel', 'cmGlobal', 'thetaLocal', 'dPanel']
        self._geometries = geometries
        self._nBodies = len(geometries)
        nPanels = []
        for name, gd in geometries.items():
            if type(gd) != dict:
                raise TypeError("geometries['%s'] must either be a dictionary, containing the "
                                "geometry's panel datas." % name)
            for k in keys:
                if k not in gd:
                    raise ValueError("%s was not found in geometries['%s']." % (k, name))
            nPanels.append(np.asarray(gd['xPanel']).shape[0] - 1)
        self._nPanels = np.array(nPanels, dtype=int)
        self._nPanelsTotal = np.int64(self._nPanels.sum())
        self._index = np.cumsum(np.hstack((0, self._nPanels)))
        self._update_coordinates()
        self._assemble()
        self._sPanel = torch.zeros(int(self._nPanelsTotal), dtype=torch.float64,
                                   device=self.device)
        self._tStep = 0
        self._t = 0.0
        self._deltaT = 0.0

    # -- geometry (host FP64, the reference's numpy operations) --------------------
    def _update_coordinates(self):
        """__panelsClass.py:1009-1058 and the rotation matrix of :1094-1096."""
        M = int(self._nPanelsTotal)
        start = np.zeros((2, M))
        end = np.zeros((2, M))
        L = np.zeros(M)
        cs = np.zeros((2, M))
        norm = np.zeros((2, M))
        tang = np.zeros((2, M))
        cp = np.zeros((2, M))
        for i, gd in enumerate(self._geometries.values()):
            th = gd['thetaLocal']
            rot = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
            iS, iE = self._index[i], self._index[i + 1]
            xy = np.dot(rot, np.vstack((gd['xPanel'], gd['yPanel']))) + \
                np.asarray(gd['cmGlobal'], dtype=np.float64).reshape(2, 1)
            start[:, iS:iE] = xy[:, :-1]
            end[:, iS:iE] = xy[:, 1:]
            Lxy = end[:, iS:iE] - start[:, iS:iE]
            L[iS:iE] = np.sqrt(np.sum(Lxy * Lxy, axis=0))
            cs[:, iS:iE] = Lxy / L[iS:iE]
            norm[:, iS:iE] = np.vstack((-cs[1, iS:iE], cs[0, iS:iE]))
            tang[:, iS:iE] = np.vstack((cs[0, iS:iE], cs[1, iS:iE]))
            cp[:, iS:iE] = 0.5 * (end[:, iS:iE] + start[:, iS:iE]) - norm[:, iS:iE] * L[iS:iE] * 0.1
        self._host = {"start": start, "end": end, "L": L, "cs": cs, "norm": norm, "tang": tang,
                      "cp": cp}
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self._d = {k: T(v) for k, v in (("xs", start[0]), ("ys", start[1]), ("xe", end[0]),
                                        ("ye", end[1]), ("cosa", cs[0]), ("sina", cs[1]),
                                        ("tx", tang[0]), ("ty", tang[1]), ("nx", norm[0]),
                                        ("ny", norm[1]), ("xcp", cp[0]),
                                        ("ycp", cp[1]))}

    def _assemble(self):
        """Influence matrix A on the device (__panelsClass.py:940-962); 'fixed':
        its LU factors; 'prescribed': the least-squares system [A; L rows] of
        __panelsClass.py:513-518, solved through its normal equations."""
        d = self._d
        M = int(self._nPanelsTotal)
        A = torch.empty((M, M), dtype=torch.float64, device=self.device)
        st = torch.cuda.current_stream(self.device).cuda_stream
        fn = _lib.lib.pf_source_panel_influence_matrix if self._panelKernel == 'css' \
            else _lib.lib.pf_panel_influence_matrix
        _lib.check(fn(_lib.context(self.device.index), M,
                      *[ptr(d[k]) for k in ("xcp", "ycp", "xs", "ys", "xe", "ye", "cosa", "sina")],
                      ptr(A), st))
        self._A = A
        if self._problemType in ('fixed', 'moving'):
            self._lu = _lu(self.device, A)
        else:
            B = torch.zeros((M + self._nBodies, M), dtype=torch.float64, device=self.device)
            B[:M] = A
            Lh = torch.from_numpy(self._host["L"]).to(self.device)
            for i in range(self._nBodies):
                B[M + i, self._index[i]:self._index[i + 1]] = Lh[self._index[i]:self._index[i + 1]]
            self._B = B
            self._lu = _lu(self.device, B.T @ B)

    # -- pHyFlow surface ------------------------------------------------------------
    def evaluateVelocity(self, xTarget, yTarget):
        """Velocity of the panels (current strengths) at the targets: CUDA
        tensors in, CUDA tensors out (numpy in, numpy out)."""
        host = not (isinstance(xTarget, torch.Tensor) and xTarget.is_cuda)
        xt = xTarget if not host else torch.from_numpy(np.ascontiguousarray(xTarget, dtype=np.float64)).to(self.device)
        yt = yTarget if not host else torch.from_numpy(np.ascontiguousarray(yTarget, dtype=np.float64)).to(self.device)
        vx, vy = torch.empty_like(xt), torch.empty_like(xt)
        self._velocity_device(xt, yt, vx, vy, accumulate=False)
        return (vx.cpu().numpy(), vy.cpu().numpy()) if host else (vx, vy)

    def _velocity_device(self, xt, yt, vx, vy, accumulate):
        d = self._d
        panel_velocity_device(self._sPanel, d["xs"], d["ys"], d["xe"], d["ye"], d["cosa"],
                              d["sina"], xt, yt, vx, vy, accumulate=accumulate,
                              panelKernel=PANEL_KERNEL_CSS if self._panelKernel == 'css'
                              else PANEL_KERNEL_CSV)

    def solve(self, vxExternel, vyExternel, gTotal=None):
        """Panel strengths for the no-slip condition at the collocation points
        under the external velocity there (RHS = -v_ext . t for vortex
        panels, -v_ext . n for source panels, __panelsClass.py:772-775)."""
        d = self._d
        vx = vxExternel if isinstance(vxExternel, torch.Tensor) else torch.from_numpy(np.asarray(vxExternel, dtype=np.float64)).to(self.device)
        vy = vyExternel if isinstance(vyExternel, torch.Tensor) else torch.from_numpy(np.asarray(vyExternel, dtype=np.float64)).to(self.device)
        if self._panelKernel == 'css':
            rhs = (-vx) * d["nx"] + (-vy) * d["ny"]
        else:
            rhs = (-vx) * d["tx"] + (-vy) * d["ty"]
        if self._problemType in ('fixed', 'moving'):
            self._sPanel = _lu_solve(self.device, *self._lu, rhs)
        else:
            if gTotal is None:
                gTotal = np.zeros(self._nBodies)
            g = torch.as_tensor(np.asarray(gTotal, dtype=np.float64), device=self.device)
            b = torch.cat([rhs, -g])
            self._sPanel = _lu_solve(self.device, *self._lu, self._B.T @ b)

    def updateBody(self, cmGlobalNew, thetaLocalNew):
        """New position and rotation of every body (dicts keyed by geometry
        key, all keys required, as __panelsClass.py:1304-1350 checks them):
        the global coordinates, normals, tangents and collocation points are
        recomputed and the influence matrix re-assembled (and re-factored)
        on the GPU (__panelsClass.py:530-637)."""
        keys = self.geometryKeys
        if type(thetaLocalNew) != dict or any(k not in thetaLocalNew for k in keys):
            raise TypeError("'thetaLocal' must either be a dictionary containing the following "
                            "keys: %s" % str(keys))
        if type(cmGlobalNew) != dict or any(k not in cmGlobalNew for k in keys):
            raise TypeError("'cmGlobal' must either be a dictionary containing the following "
                            "keys: %s" % str(keys))
        for k in keys:
            if type(thetaLocalNew[k]) not in (float, np.float64):
                raise TypeError("thetaLocal['%s'] must be a float. It is a %s"
                                % (k, type(thetaLocalNew[k])))
            cm = np.asarray(cmGlobalNew[k], dtype=np.float64)
            if cm.shape != (2,):
                raise ValueError("cmGlobal['%s'] must have shape (2,). It has shape %s."
                                 % (k, str(cm.shape)))
        for k in keys:  # thetaLocal first, then cmGlobal, as the reference sets them
            self._geometries[k]['thetaLocal'] = thetaLocalNew[k]
        for k in keys:
            self._geometries[k]['cmGlobal'] = np.asarray(cmGlobalNew[k], dtype=np.float64)
        self._update_coordinates()
        self._assemble()

    def _advanceTime(self, deltaTNew):
        """__panelsClass.py:825-870: deltaT kept, tStep + 1, t = deltaT tStep."""
        self._deltaT = deltaTNew
        self._tStep += 1
        self._t = self._deltaT * self._tStep

    # -- properties ---------------------------------------------------------------------
    @property
    def sPanel(self):
        return self._sPanel.cpu().numpy()

    @property
    def A(self):
        return self._A.cpu().numpy()

    @property
    def nPanelsTotal(self):
        return self._nPanelsTotal

    @property
    def geometryKeys(self):
        return list(self._geometries.keys())

    @property
    def cmGlobal(self):
        """Per body, as __panelsClass.py:1365-1373 (a list in body order)."""
        return [np.asarray(gd['cmGlobal'], dtype=np.float64).copy()
                for gd in self._geometries.values()]

    @property
    def thetaLocal(self):
        return [gd['thetaLocal'] for gd in self._geometries.values()]

    def _per_body(self, a):
        """([a[0] of body i], [a[1] of body i]) (the reference's per-body lists)."""
        ix = self._index
        return ([a[0, ix[i]:ix[i + 1]].copy() for i in range(self._nBodies)],
                [a[1, ix[i]:ix[i + 1]].copy() for i in range(self._nBodies)])

    @property
    def normCat(self):
        return self._host["norm"].copy()

    @property
    def tangCat(self):
        return self._host["tang"].copy()

    @property
    def xyCPGlobal(self):
        return self._per_body(self._host["cp"])

    @property
    def xyPanelGlobal(self):
        """Per body, closed: its start points and its first start point again."""
        xs, ys = self._per_body(self._host["start"])
        return [np.append(a, a[0]) for a in xs], [np.append(a, a[0]) for a in ys]

    @property
    def xyPanelLocal(self):
        return ([np.asarray(gd['xPanel']) for gd in self._geometries.values()],
                [np.asarray(gd['yPanel']) for gd in self._geometries.values()])

    @property
    def gTotal(self):
        """Total circulation of each body, sum(-gamma L) (__panelsClass.py);
        zero for source panels."""
        if self._panelKernel == 'css':
            return np.zeros(self._nBodies)
        s, L, ix = self.sPanel, self._host["L"], self._index
        return [np.sum(-s[ix[i]:ix[i + 1]] * L[ix[i]:ix[i + 1]]) for i in range(self._nBodies)]

    @property
    def velCompParams(self):
        return dict(self._velCompParams)

    @property
    def deltaT(self):
        return self._deltaT

    @property
    def solverCompParams(self):
        return dict(self._solverCompParams)

    @property
    def nPanels(self):
        return self._nPanels

    @property
    def nBodies(self):
        return self._nBodies

    @property
    def xyCPGlobalCat(self):
        return self._host["cp"].copy()

    @property
    def xyPanelGlobalCat(self):
        """(2, nPanelsTotal + nBodies): each body's start points closed by its
        first start point."""
        xs, ys = self.xyPanelGlobal
        return np.vstack((np.concatenate(xs), np.concatenate(ys)))

    @property
    def norm(self):
        """Per body, as __panelsClass.py:1400-1409; normCat is the (2, M) array."""
        return self._per_body(self._host["norm"])

    @property
    def tang(self):
        return self._per_body(self._host["tang"])

    @property
    def t(self):
        return self._t

    @property
    def tStep(self):
        return self._tStep

    @property
    def problemType(self):
        return self._problemType

    @property
    def panelKernel(self):
        return self._panelKernel


class LagrangianSolver:
    """Blobs coupled with vortex panels (no-through-flow on the bodies)."""

    def __init__(self, blobs, panels=None, couplingParams={'panelStrengthUpdate': 'constant'}):
        if couplingParams.get('panelStrengthUpdate') not in PANEL_STRENGTH_UPDATES:
            raise ValueError("couplingParams['panelStrengthUpdate'] must be one of %s"
                             % str(PANEL_STRENGTH_UPDATES))
        self.blobs = blobs
        self.panels = panels
        self._couplingParams = dict(couplingParams)
        if self.panels is not None:
            self._solve_panelStrength()

    @property
    def couplingParams(self):
        return dict(self._couplingParams)

    @property
    def vInf(self):
        return np.asarray(self.blobs.vInf, dtype=np.float64)

    @property
    def deltaT(self):
        return self.blobs.deltaTc

    @property
    def t(self):
        return self.blobs.t

    @property
    def tStep(self):
        return self.blobs.tStep

    def _method(self):
        return FMM_METHOD if self.blobs.velocityComputationParams['method'] == 'fmm' \
            else DIRECT_METHOD

    def _blob_velocity(self, x, y, g, xt, yt):
        """Blob-induced velocity at (xt, yt) with the blobs at (x, y):
        ``velocity`` with its defaults (tol 1e-6, Ndirect 35), as the
        reference's ``_blobs_velocity`` calls are made."""
        ks, xo, cut = fmm_parameters(self.blobs.sigma, 2.0)
        vx, vy = torch.empty_like(xt), torch.empty_like(xt)
        velocity_device(x, y, g, ks, xt, yt, vx, vy, method=self._method(), xopt=xo, cutoff=cut)
        return vx, vy

    def _slip_solve(self, x, y):
        """Panel strengths from the blob + free-stream velocity at the
        collocation points (__lagrangianSolverClass.py:439-445, 611-636)."""
        d = self.panels._d
        vx, vy = self._blob_velocity(x, y, self.blobs._g, d["xcp"], d["ycp"])
        self.panels.solve(vx + self.vInf[0], vy + self.vInf[1])

    def _solve_panelStrength(self):
        self._slip_solve(self.blobs._x, self.blobs._y)

    def evaluateVelocity(self, xTarget, yTarget, Ndirect=35, tol=1.0e-6, cutoff=None):
        """Blob + panel + free-stream velocity at the targets
        (__lagrangianSolverClass.py:245-263)."""
        host = not (isinstance(xTarget, torch.Tensor) and xTarget.is_cuda)
        dev = self.blobs.device
        xt = xTarget if not host else torch.from_numpy(np.ascontiguousarray(xTarget, dtype=np.float64)).to(dev)
        yt = yTarget if not host else torch.from_numpy(np.ascontiguousarray(yTarget, dtype=np.float64)).to(dev)
        ks, xo, cut = fmm_parameters(self.blobs.sigma, 2.0, cutoff, tol)
        vx, vy = torch.empty_like(xt), torch.empty_like(xt)
        b = self.blobs
        velocity_device(b._x, b._y, b._g, ks, xt, yt, vx, vy, method=self._method(), xopt=xo,
                        cutoff=cut, tol=tol, ndirect=Ndirect)
        if self.panels is not None:
            self.panels._velocity_device(xt, yt, vx, vy, accumulate=True)
        vx = vx + self.vInf[0]
        vy = vy + self.vInf[1]
        return (vx.cpu().numpy(), vy.cpu().numpy()) if host else (vx, vy)

    def evolve(self):
        """One step (__lagrangianSolverClass.py:341-368): without panels,
        ``blobs.evolve()``; with panels, the coupled convection, diffusion,
        time advance, redistribution and population control."""
        b = self.blobs
        if self.panels is None:
            b.evolve()
            return
        self._coupled_convection()
        if b.stepDiffusion != 0 and (b.tStep % b.stepDiffusion) == 0:
            b._diffusion()
        self._advanceTime()
        if b.stepRedistribution != 0 and (b.tStep % b.stepRedistribution) == 0:
            b.redistribute()
        if b.stepPopulationControl != 0 and (b.tStep % b.stepPopulationControl) == 0:
            b.populationControl()

    def _advanceTime(self):
        self.blobs._advanceTime()
        self.panels._advanceTime(self.deltaT)
        if abs(self.blobs.t - self.panels.t) > np.spacing(100):
            raise ValueError('The internal time of Blobs and Panels are not synchronized. '
                             'blobs = %g, panels = %g' % (self.blobs.t, self.panels.t))

    def _coupled_convection(self):
        """The coupled RK4 of __lagrangianSolverClass.py:586-677 (forward Euler
        raises there, :679-680).  The positions are updated in place after each
        stage, as the reference's are (see the module docstring)."""
        b = self.blobs
        if b.timeIntegrationParams['method'] != 'rk4':
            raise NotImplementedError('FE time integration not available !')
        dt = self.deltaT
        x, y, g = b._x, b._y, b._g  # updated in place below, as the reference's arrays are
        vinf = self.vInf
        kx = ky = None
        update = self._couplingParams['panelStrengthUpdate']
        for stage, rb, rc in zip((1, 2, 3, 4), (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0),
                                 (0.0, 0.5, 0.5, 1.0)):
            if kx is None:  # k = 0: the temporary positions are the positions
                xt, yt = x.clone(), y.clone()
            else:
                xt, yt = x + (rc * dt) * kx, y + (rc * dt) * ky
            if update == 'varying' or stage == 1:
                self._slip_solve(xt, yt)
            vxp, vyp = torch.empty_like(xt), torch.empty_like(xt)
            self.panels._velocity_device(xt, yt, vxp, vyp, accumulate=False)
            vxb, vyb = self._blob_velocity(xt, yt, g, xt, yt)
            kx = (vxb + vxp) + vinf[0]
            ky = (vyb + vyp) + vinf[1]
            x += (rb * kx) * dt
            y += (rb * ky) * dt
