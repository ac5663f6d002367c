"""B200-native spectral placement for SpectraPack (nesickc/cpp-max-packer).

The hot path - rasterise, FFT-correlate, threshold, reduce, stamp - runs as
hand-written sm_100a CUDA kernels behind the C ABI in include/spk_b200.h;
this package is the host-side mirror of the reference's interfaces for that
path (compute::correlate_*, build_proximity, the spectral pipeline pages and
the greedy placement loop).  There is no CPU fallback.
"""

from . import _lib  # noqa: F401
from ._lib import SpkError, SpkUnavailable  # noqa: F401
