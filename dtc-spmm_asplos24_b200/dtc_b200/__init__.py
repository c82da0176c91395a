"""B200-native DTC-SpMM: ME-TCF conversion + tcgen05 TC-block SpMM.

The reference-compatible module is ``DTCSpMM`` (built next to this package);
this package is the Python front end over the same C ABI (libdtcspmm.so):
``metcf`` (conversion / SpMM on torch tensors), ``gen`` (seeded synthetic
inputs).
"""
from . import _lib  # noqa: F401
from ._lib import (B_BF16, B_BF16X2, B_F32, B_FP8, B_SPLIT24,  # noqa: F401
                   PREC_SPLIT3, PREC_SPLIT4,
                   PREC_TF32, DtcError)
