"""``Blobs``: the vortex-blob state object with pHyFlow's call surface, the
blob set resident on the GPU.

Keeps the constructor arguments, parameter dictionaries, methods and
properties of ``pHyFlow.blobs.Blobs`` (``src/python/blobs/__blobsClass.py``)
that touch the hot path: ``evaluateVelocity`` (:546-628), ``redistribute``
(:828-897), ``populationControl`` (:783-825), ``addBlobs`` / ``removeBlobs``
(:499-544, :900-960), the construction-time population control and
redistribution (:490-494), and ``evolve`` (:705-781) with the reference's
convection integrators (``_evolution.py:537-701``) and Wee or Tutty diffusion
(``_evolution.py:138-445``, ``_diffusion`` :1002-1111, time step from
``__compute_deltaTd`` :2248-2318).
Properties return numpy copies, as the reference's numpy-backed object does,
and are read-only where the reference's are (:2324-3020): setting or deleting
one raises AttributeError; ``vInf``, ``hardware`` and ``plotVelocity`` can be
set.  ``evaluateVorticity`` is kept as the reference has it (:631-703, a method
without a body that returns None); the induced vorticity itself is
``pfblob.vorticity``.
"""
import math

import numpy as np
import torch

from .evolution import FE_INTEGRATOR, RK4_INTEGRATOR, convection_device
from .induced import DIRECT_METHOD, FMM_METHOD, fmm_parameters, velocity_device
from .regrid import population_control_device, remesh_device

default_diffusion_params = {'method': 'regrid_wee', 'c2': 'optimized'}
default_time_integration_params = {'method': 'rk4'}
default_blob_control_params = {'stepRedistribution': 1, 'stepPopulationControl': 1,
                               'gThresholdLocal': 1e-8, 'gThresholdGlobal': 1e-8}
default_velocity_computation_params = {'method': 'fmm', 'hardware': 'gpu'}


def _round_half_away(r):
    """Nearest integer to r >= 0, halves away from zero: the rounding of the
    reference's Python-2 ``round`` (Python 3's rounds halves to even, so a
    ratio of exactly 2.5 would give 2 instead of the reference's 3)."""
    q = math.floor(r)
    return int(q) + (1 if r - q >= 0.5 else 0)


def _read_only(name, attr=None):
    """Property returning self.<attr> (default _<name>); setting or deleting it
    raises AttributeError with the reference's message."""
    attr = attr or "_" + name

    def get(self):
        return getattr(self, attr)

    def set_(self, value):
        raise AttributeError('%s cannot be manually set by the user, user can only get the value '
                             'of %s.' % (name, name))

    def del_(self):
        raise AttributeError('%s cannot be manually deleted by the user, user can only get the '
                             'value of %s.' % (name, name))

    return property(get, set_, del_)


HARDWARE_OPTIONS = ('cpu', 'gpu')


class Blobs:
    def __init__(self, wField, vInf, nu, deltaTc, h, overlap,
                 timeIntegrationParams=default_time_integration_params,
                 blobControlParams=default_blob_control_params,
                 velocityComputationParams=default_velocity_computation_params,
                 diffusionParams=default_diffusion_params, device=None):
        if len(wField) != 3:
            raise ValueError("wField must have exactly 3 arrays. It has %d." % len(wField))
        self.device = self._device_for(device)
        if callable(wField[0]):
            x, y, g = self._blobs_from_function(wField, h)
        else:
            x, y, g = (np.asarray(a, dtype=np.float64).ravel() for a in wField)
            if not (x.shape == y.shape == g.shape):
                raise ValueError("wField arrays must have the same shape")
        self._x, self._y, self._g = (self._dev(a) for a in (x, y, g))
        self._vInf = np.asarray(vInf, dtype=np.float64)
        self._nu = float(nu)
        self._deltaTc = float(deltaTc)
        self._h = float(h)
        self._overlap = float(overlap)
        self._sigma = self._h / self._overlap
        self._timeIntegrationParams = dict(timeIntegrationParams)
        self._blobControlParams = dict(blobControlParams)
        self._velocityComputationParams = dict(velocityComputationParams)
        self._diffusionParams = dict(diffusionParams)
        if self.timeIntegrationParams['method'] not in ('euler', 'rk4'):
            raise ValueError("timeIntegrationParams['method'] must be 'euler' or 'rk4'")
        if self.velocityComputationParams['method'] not in ('fmm', 'direct'):
            raise ValueError("velocityComputationParams['method'] must be 'fmm' or 'direct'")
        if self.velocityComputationParams.get('hardware', 'gpu') not in HARDWARE_OPTIONS:
            raise ValueError("velocityComputationParams['hardware'] must be 'cpu' or 'gpu'")
        if self.diffusionParams['method'] not in ('regrid_wee', 'regrid_tutty'):
            raise ValueError("diffusionParams['method'] must be 'regrid_wee' or 'regrid_tutty'")
        self._deltaTd, self._stepDiffusion = self._compute_deltaTd()
        self._tStep = 0
        self._t = 0.0
        self._plotVelocity = False
        if self.stepPopulationControl > 0:
            self.populationControl()
        if self.stepRedistribution > 0:
            self.redistribute()

    # -- helpers ----------------------------------------------------------------
    @staticmethod
    def _device_for(device):
        """The CUDA device holding the blob set (the current one if None)."""
        return torch.device("cuda", torch.cuda.current_device() if device is None else device)

    def _dev(self, a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self.device)

    def _blobs_from_function(self, wField, h):
        """(wExactFunction, xBounds, yBounds): floor(width / h) blobs per
        direction at the cell centres xBounds[0] + h/2 + i h, x varying
        fastest, circulation w(x, y) h^2 -- the reference's
        ``__read_input_wField_function`` (``__blobsClass.py:1406-1419``)."""
        f, xb, yb = wField
        nx = int(np.floor((xb[1] - xb[0]) / h))
        ny = int(np.floor((yb[1] - yb[0]) / h))
        xs = xb[0] + 0.5 * h + np.arange(0, nx) * h
        ys = yb[0] + 0.5 * h + np.arange(0, ny) * h
        X, Y = np.meshgrid(xs, ys)
        x, y = X.flatten(), Y.flatten()
        return x, y, f(x, y) * h * h

    def _compute_deltaTd(self):
        """Diffusion time step and interval (__blobsClass.py:2248-2318): Wee
        rounds the stable step to a multiple of deltaTc; Tutty diffuses every
        step and needs hNu/h <= 1/sqrt(2)."""
        if self.nu == 0.0:
            return 0.0, 0
        if self.diffusionParams['method'] == 'regrid_tutty':
            deltaTd = self.deltaTc
            hnu = np.sqrt(deltaTd * self.nu)
            if ((hnu / self.h) - (1.0 / np.sqrt(2.0))) > np.spacing(1000):
                deltaTd = (((1.0 / np.sqrt(2.0)) * self.h) ** 2) / self.nu
                raise ValueError('Regrid Tutty: deltaTc is to large. Reduce deltaTc to a value '
                                 'smaller than %f.' % deltaTd)
            return deltaTd, 1
        c2 = self.diffusionParams['c2']
        deltaTd = ((1.0 / 3.0) * self.h * self.h) / self.nu if c2 == 'optimized' else \
            (float(c2) * self.h * self.h) / self.nu
        if deltaTd >= self.deltaTc:
            step = _round_half_away(deltaTd / self.deltaTc)
            return step * self.deltaTc, step
        raise ValueError('Regrid Wee: deltaTc is too large. Reduce deltaTc to a value smaller '
                         'than %f.' % deltaTd)

    def _method(self):
        return FMM_METHOD if self.velocityComputationParams['method'] == 'fmm' else DIRECT_METHOD

    def _velocity_at(self, xs, ys, xt, yt, Ndirect=35, tol=1.0e-6, cutoff=None):
        ks, xo, cut = fmm_parameters(self.sigma, 2.0, cutoff, tol)
        vx = torch.empty_like(xt)
        vy = torch.empty_like(xt)
        velocity_device(xs, ys, self._g, ks, xt, yt, vx, vy, method=self._method(), xopt=xo,
                        cutoff=cut, tol=tol, ndirect=Ndirect)
        return vx, vy

    def _regrid(self, c, population_control=False, tutty_hnu=None):
        # The reference passes (sigma, overlap) to Regrid, which remeshes with
        # h = sigma*overlap (_regridding.py:118), and bounds -1.5 h from the
        # stored h (__blobsClass.py:891-892); the two can differ in the last bit.
        h = self.sigma * self.overlap
        b0 = -1.5 * self.h
        if tutty_hnu is not None:
            self._x, self._y, self._g = remesh_device(self._x, self._y, self._g, h, b0, b0,
                                                      tutty_hnu=tutty_hnu)
        elif population_control:
            self._x, self._y, self._g, _ = remesh_device(
                self._x, self._y, self._g, h, b0, b0, c,
                population_control=(self.gThresholdLocal, self.gThresholdGlobal))
        else:
            self._x, self._y, self._g = remesh_device(self._x, self._y, self._g, h, b0, b0, c)

    # -- hot-path methods ---------------------------------------------------------
    def evaluateVelocity(self, xEval=None, yEval=None, Ndirect=35, tol=1.0e-6, cutoff=None):
        """Induced velocity at (xEval, yEval) (the blobs if None); numpy in and
        out, or CUDA tensors in and out."""
        if xEval is None:
            xt, yt, host = self._x, self._y, True
        else:
            host = not isinstance(xEval, torch.Tensor)
            xt = xEval.to(self.device, torch.float64).contiguous() if not host else self._dev(xEval)
            yt = yEval.to(self.device, torch.float64).contiguous() if not host else self._dev(yEval)
        vx, vy = self._velocity_at(self._x, self._y, xt, yt, Ndirect, tol, cutoff)
        return (vx.cpu().numpy(), vy.cpu().numpy()) if host else (vx, vy)

    def evaluateVorticity(self, xEval, yEval):
        """The reference's method has no body and returns None
        (``__blobsClass.py:631-703``); kept so that code calling it behaves the
        same.  The induced vorticity is ``pfblob.vorticity``."""
        return None

    def redistribute(self, interpKernel=0):
        """M4' remesh onto the lattice containing (0, 0) (xBounds = [-1.5h, 1.5h])."""
        if interpKernel != 0:
            raise NotImplementedError("pfblob: only the M4' kernel (interpKernel=0) exists")
        if self.numBlobs > 0:
            self._regrid(0.0)

    def populationControl(self):
        """Drop blobs with |g| below gThresholdLocal while the dropped
        circulation stays below gThresholdGlobal (threshold /10 otherwise),
        as PopulationControl (_regridding.py:227-330), on the device
        (pf_population_control)."""
        self._x, self._y, self._g, _ = population_control_device(
            self._x, self._y, self._g, self.gThresholdLocal, self.gThresholdGlobal)

    def evolve(self):
        """One time step: convection (FE or the reference's RK4), diffusion
        (Wee every stepDiffusion steps, or Tutty every step), redistribution
        and population control.  With Wee and nu = 0 the reference divides by
        stepDiffusion = 0; here diffusion is skipped."""
        # convection (_evolution.py:37-135): forward Euler, or the reference's
        # RK4, whose four stages all sit at the start positions
        integrator = FE_INTEGRATOR if self.integrationMethod == 'euler' else RK4_INTEGRATOR
        self._x, self._y = convection_device(self.deltaTc, self._x, self._y, self._g, self.sigma,
                                             2.0, self.vInf, self._method(), integrator)
        self._diffusion()
        redistribute = self.stepRedistribution != 0 and (self.tStep % self.stepRedistribution) == 0
        control = (self.stepPopulationControl != 0 and
                   ((self.tStep + 1) % self.stepPopulationControl) == 0)
        # redistribution followed by population control (after the time
        # advance, which does not touch the blobs) runs as one fused remesh
        fused = redistribute and control and self.numBlobs > 0
        if fused:
            self._regrid(0.0, population_control=True)
        elif redistribute:
            self.redistribute()
        self._advanceTime()
        if control and not fused:
            self.populationControl()

    def _diffusion(self):
        """Diffusion step (__blobsClass.py:1002-1111): Wee's diffusive remesh
        every stepDiffusion steps, or -- with 'regrid_tutty' -- a
        redistribution followed by Tutty's diffusive redistribution, every
        call (hNu = 0 when nu = 0)."""
        if self.diffusionParams['method'] == 'regrid_tutty':
            self.redistribute()
            if self.numBlobs > 0:
                self._regrid(0.0, tutty_hnu=float(np.sqrt(self.deltaTd * self.nu)))
        elif self.stepDiffusion != 0 and (self.tStep % self.stepDiffusion) == 0:
            self._regrid(math.sqrt(self.nu * self.deltaTd) / self.h)

    def _advanceTime(self):
        """tStep + 1 and t = deltaTc * tStep, as the reference's _advanceTime
        (a product, not a running sum)."""
        self._tStep += 1
        self._t = self.deltaTc * self._tStep

    def addBlobs(self, xNew, yNew, gNew):
        self._x = torch.cat([self._x, self._dev(xNew)])
        self._y = torch.cat([self._y, self._dev(yNew)])
        self._g = torch.cat([self._g, self._dev(gNew)])

    def removeBlobs(self, iBlobs):
        """As the reference's ``removeBlobs`` (``__blobsClass.py:935-955``):
        an int64 array lists the blobs to delete; a bool array of numBlobs
        entries selects the blobs to KEEP (the reference indexes with it);
        anything else raises TypeError."""
        if type(iBlobs) != np.ndarray:
            raise TypeError('iBlobs must be a numpy.array, it is a %s.' % str(type(iBlobs)))
        if iBlobs.dtype == np.dtype('int64'):
            if iBlobs.size and iBlobs.max() >= self.numBlobs:
                raise TypeError('iBlobs values must be smaller than the numBlobs: %d.'
                                % self.numBlobs)
            keep = np.ones(self.numBlobs, dtype=bool)
            keep[iBlobs] = False  # numpy.delete: negative indices count from the end
        elif iBlobs.dtype == np.dtype('bool'):
            if iBlobs.shape != (self.numBlobs,):
                raise TypeError('iBlobs of type bool must have as many elements as numBlobs: %d.'
                                % self.numBlobs)
            keep = iBlobs
        else:
            raise TypeError('iBlobs must be of type int64 or bool, it is a %s.' % str(iBlobs.dtype))
        k = torch.from_numpy(np.ascontiguousarray(keep)).to(self.device)
        self._x, self._y, self._g = self._x[k], self._y[k], self._g[k]

    # -- properties ---------------------------------------------------------------
    # read-only unless noted, with the reference's AttributeError messages
    h = _read_only("h")
    sigma = _read_only("sigma")
    overlap = _read_only("overlap")
    deltaTc = _read_only("deltaTc")
    deltaTd = _read_only("deltaTd")
    nu = _read_only("nu")
    tStep = _read_only("tStep")
    t = _read_only("t")
    stepDiffusion = _read_only("stepDiffusion")
    diffusionParams = _read_only("diffusionParams")
    timeIntegrationParams = _read_only("timeIntegrationParams")
    blobControlParams = _read_only("blobControlParams")
    velocityComputationParams = _read_only("velocityComputationParams")
    x = _read_only("x", "_x_host")
    y = _read_only("y", "_y_host")
    g = _read_only("g", "_g_host")
    numBlobs = _read_only("numBlobs", "_num_blobs")
    stepRedistribution = _read_only("stepRedistribution", "_step_redistribution")
    stepPopulationControl = _read_only("stepPopulationControl", "_step_population_control")
    gThresholdLocal = _read_only("gThresholdLocal", "_g_threshold_local")
    gThresholdGlobal = _read_only("gThresholdGlobal", "_g_threshold_global")
    integrationMethod = _read_only("integrationMethod", "_integration_method")
    computationMethod = _read_only("computationMethod", "_computation_method")

    @property
    def _x_host(self):
        return self._x.cpu().numpy()

    @property
    def _y_host(self):
        return self._y.cpu().numpy()

    @property
    def _g_host(self):
        return self._g.cpu().numpy()

    @property
    def _num_blobs(self):
        return self._x.numel()

    @property
    def _step_redistribution(self):
        return int(self.blobControlParams['stepRedistribution'])

    @property
    def _step_population_control(self):
        return int(self.blobControlParams['stepPopulationControl'])

    @property
    def _g_threshold_local(self):
        return float(self.blobControlParams['gThresholdLocal'])

    @property
    def _g_threshold_global(self):
        return float(self.blobControlParams['gThresholdGlobal'])

    @property
    def _integration_method(self):
        return self.timeIntegrationParams['method']

    @property
    def _computation_method(self):
        return self.velocityComputationParams['method']

    @property
    def vInf(self):
        return self._vInf

    @vInf.setter
    def vInf(self, vInfnew):
        v = np.asarray(vInfnew, dtype=np.float64)
        if v.shape != (2,):
            raise ValueError('vInf must have shape (2,0). It has shape %s.' % str(v.shape))
        self._vInf = v

    @vInf.deleter
    def vInf(self):
        raise AttributeError('vInf cannot be manually deleted by the user, user can only get the '
                             'value of vInf.')

    @property
    def hardware(self):
        """'cpu' or 'gpu' as given; every computation here runs on the GPU."""
        return self.velocityComputationParams['hardware']

    @hardware.setter
    def hardware(self, hardwarenew):
        if hardwarenew not in HARDWARE_OPTIONS:
            raise ValueError("velocityComputationParams['hardware'] must be 'cpu' or 'gpu'")
        self.velocityComputationParams['hardware'] = hardwarenew

    @hardware.deleter
    def hardware(self):
        raise AttributeError('hardware cannot be deleted by the user, user can only get and set '
                             'the value of hardware.')

    @property
    def plotVelocity(self):
        return self._plotVelocity

    @plotVelocity.setter
    def plotVelocity(self, plotVelocitynew):
        if type(plotVelocitynew) != bool:
            raise TypeError('plotVelocity must be of type bool. It is of type: %s'
                            % str(type(plotVelocitynew)))
        self._plotVelocity = plotVelocitynew

    @plotVelocity.deleter
    def plotVelocity(self):
        raise AttributeError('plotVelocity cannot be deleted by the user, user can only get and set '
                             'the value of plotVelocity.')
