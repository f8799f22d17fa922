"""FP64 CPU oracle for the pHyFlow vortex-blob hot path.

TEST INFRASTRUCTURE ONLY.  This package is the checker: the parity tests in
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import it to compute the FP64 answer (and, for the baseline, to
time the reference's CPU code).  The product package never imports it and has
no CPU fallback.

Contents
--------
``liboracle.so`` (built from ``pf_oracle.c``)
    our C restatement of the reference kernels: direct Gauss velocity, vortex
    panel velocity, M4' weights, remesh window indices, FP64 moments.
``regrid``
    the remesh (``Regrid``) restated in numpy + scipy.sparse, following
    ``src/python/blobs/base/regrid/_regridding.py:107-222``.
``lists``
    a CPU restatement of the FMM box-pair rule of this library, used to check
    the interaction lists the library builds bit for bit.
``ref``
    loaders for the reference's own CPU code compiled in place from the
    pHyFlow sources into ``oracle/_ref/`` (Cython direct Gauss, Cython vortex
    panels, the C++ CPU FMM).  These pin the restatement.
"""
from .core import (velocity_direct, vorticity_direct, velocity_direct_cutoff,
                   vorticity_direct_cutoff, panel_velocity, source_panel_velocity, m4prime,
                   remesh_left_index, moments, oracle_lib)
from .regrid import diffusion_tutty, population_control, regrid

__all__ = ["velocity_direct", "vorticity_direct", "velocity_direct_cutoff",
           "vorticity_direct_cutoff", "panel_velocity", "source_panel_velocity", "m4prime",
           "remesh_left_index",
           "moments", "regrid", "population_control", "diffusion_tutty", "oracle_lib"]
