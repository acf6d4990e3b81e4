"""dirac_b200: B200 (sm_100a) implementation of the Dirac research codec's data-parallel
coding hot path, reached through the C ABI in include/dirac_gpu.h."""
from . import _lib
from ._lib import DgpuError, load
from .wavelet import (BACKWARD, DAUB9_7, DD9_7, DD13_7, FIDELITY, FILTER_NAMES, FORWARD,
                      HAAR0, HAAR1, LEGALL5_3, WaveletTransform, padded_size, transform_batch)
from . import motion, quant, synth
from .motion import BlockParams, MotionCompensator, MotionEstimator, clip, downconvert, upconvert
