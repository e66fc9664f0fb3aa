"""hpvcd_b200 -- B200-native reconstruction back end for the hpvcd HEVC/HEIC decoder.

The host keeps demux, parameter sets, CABAC and syntax decode; this package
takes the flat per-picture buffers that syntax decode produces and runs
dequantisation, inverse transforms, intra prediction, motion compensation,
deblocking, SAO and YCbCr->RGB on the GPU through the C ABI in
include/hpvcd_gpu.h (libhpvcd_b200.so).
"""
from . import abi  # noqa: F401

__all__ = ["abi"]
