"""pfblob -- B200-native vortex-blob hot path with pHyFlow's Python call surface.

Entry points (same names, arguments and results as pHyFlow):

* ``velocity``         - pHyFlow.blobs.base.induced.velocity (direct / FMM, Gauss)
* ``vorticity``        - pHyFlow.blobs.base.induced.vorticity (direct, Gauss)
* ``Regrid``           - pHyFlow.blobs.base.regrid.Regrid (M4' remesh)
* ``velocity_and_regrid`` - ``velocity`` then ``Regrid`` of the same blobs from one upload
* ``PopulationControl`` - pHyFlow.blobs.base.regrid.PopulationControl
* ``convection``, ``diffusion_wee``, ``diffusion_tutty`` - pHyFlow.blobs.base.evolution
* ``inducedVelocity``, ``influenceMatrix`` - pHyFlow.panels.base.panelSolver
* ``lu_factor``, ``lu_solve`` - the panel-strength solve of pHyFlow.panels.Panels
* ``Blobs``            - the evaluateVelocity / redistribute surface of pHyFlow.blobs.Blobs
* ``Panels``, ``LagrangianSolver`` - fixed vortex-panel bodies and the coupled
  blob + panel step of pHyFlow.panels.Panels / pHyFlow.lagrangian.LagrangianSolver
* ``StepGraph``        - a resident set's velocity + remesh step as one CUDA graph
  launch (no pHyFlow counterpart)

All computation runs in libpfblob.so (hand-written CUDA for sm_100a) through
the C ABI of include/pfblob.h; PyTorch provides device buffers and streams.
"""
from . import _lib
from .blobs import Blobs
from .conservation import conservation_error, moments_device
from .diffusion import diffusion_tutty, diffusion_wee
from .evolution import convection, convection_device
from .lagrangian import LagrangianSolver, Panels
from .induced import (CPU_HARDWARE, DIRECT_METHOD, FMM_METHOD, GAUSS_KERNEL, GPU_HARDWARE,
                      fmm_parameters, velocity, velocity_device, vorticity)
from .panels import inducedVelocity, influenceMatrix, lu_factor, lu_solve, panel_velocity_device
from .regrid import (PopulationControl, Regrid, population_control_device, remesh_device,
                     remesh_device_async, velocity_and_regrid)
from .stepgraph import StepGraph

__all__ = ["Blobs", "Panels", "LagrangianSolver", "StepGraph", "velocity", "velocity_device", "vorticity", "Regrid", "remesh_device",
           "remesh_device_async", "velocity_and_regrid", "PopulationControl",
           "population_control_device", "convection", "convection_device", "diffusion_wee",
           "diffusion_tutty", "inducedVelocity",
           "influenceMatrix", "lu_factor", "lu_solve",
           "panel_velocity_device", "moments_device", "conservation_error", "fmm_parameters",
           "GAUSS_KERNEL", "CPU_HARDWARE", "GPU_HARDWARE", "FMM_METHOD", "DIRECT_METHOD"]

version = _lib.version
