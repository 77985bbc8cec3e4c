"""B200-native batched trajectory similarity (DTW, EDR, LCSS, ERP, discrete
Frechet, Hausdorff): hand-written sm_100a kernels behind a C ABI
(include/tsm.h), with the reference's Python call surface in ``core``."""
from . import _lib  # noqa: F401

__version__ = "0.1.0"
