"""FP64 circulation / linear-impulse checks on the device (``pf_moments``)."""
import ctypes

import torch

from . import _lib
from ._arrays import ptr, require


def moments_device(x, y, g, out=None, stream=None):
    """Device tensor [sum g, sum g x, sum g y, sum |g|] (fixed reduction order)."""
    dev = x.device
    require(x.numel(), dev, x=x, y=y, g=g)
    if out is None:
        out = torch.empty(4, dtype=torch.float64, device=dev)
    require(4, dev, out=out)
    st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream if stream is None else stream)
    _lib.check(_lib.lib.pf_moments(_lib.context(dev.index), x.numel(), ptr(x), ptr(y), ptr(g),
                                   ptr(out), st))
    return out


def conservation_error(before, after, xscale):
    """Relative circulation and impulse change between two moment vectors:
    |dG| / sum|g|  and  max(|dIx|, |dIy|) / (sum|g| * xscale)."""
    b = [float(v) for v in before]
    a = [float(v) for v in after]
    den = b[3] if b[3] > 0 else 1.0
    circ = abs(a[0] - b[0]) / den
    imp = max(abs(a[1] - b[1]), abs(a[2] - b[2])) / (den * (xscale if xscale > 0 else 1.0))
    return circ, imp
