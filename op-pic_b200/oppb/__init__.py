"""oppb — B200 particle hot path of an unstructured-mesh PIC step (Python host side).

The compute runs in liboppb.so (hand-written sm_100a CUDA, C ABI in include/oppb.h);
this package only owns device buffers and sequences the calls.
"""
from . import _lib
from ._lib import OppbError, load

__all__ = ["OppbError", "load", "_lib"]
