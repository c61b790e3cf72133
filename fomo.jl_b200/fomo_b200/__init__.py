"""fomo_b200 -- Fomo.jl's time-stepping solvers on B200 (sm_100a) via libfomo_b200.so.

Python mirror of the reference's public API (acoustic2d, elastic2d, scalar2d,
the _batch variants, acoustic3d, elastic3d and coupled2d) over the C ABI in include/fomo_b200.h.  The CUDA
library is the only compute path; there is no CPU fallback.
"""
from ._lib import FomoError, context, lib  # noqa: F401
from .api import (  # noqa: F401
    ArgumentError,
    acoustic2d,
    acoustic3d,
    acoustic2d_batch,
    acoustic2d_uneven,
    coupled2d,
    debug_coupled_medium,
    debug_medium2d,
    elastic2d,
    elastic2d_batch,
    elastic3d,
    get_centered_d2,
    get_fd_coefficients,
    ricker_wavelet,
    scalar2d,
)

__version__ = "0.1.0"
