"""hiparti_b200 -- sparse MTTKRP (COO / HiCOO) and CPD-ALS on NVIDIA B200.

A from-scratch sm_100a implementation of the MTTKRP / CPD-ALS path of HiParTI
behind the reference's C API (libhiparti_b200.so, include/hiparti_b200.h).
This package is the Python face of that library: cffi bindings generated from
the header, numpy-backed host tensors, and torch-facing device tensors.
"""
from ._ffi import PtiError, ffi, last_error, lib
from .api import COOTensor, DeviceTensor, HiCOOTensor, dump_kruskal, load_cpd_checkpoint

__all__ = ["COOTensor", "HiCOOTensor", "DeviceTensor", "PtiError", "ffi", "lib", "last_error",
           "load_cpd_checkpoint", "dump_kruskal"]
