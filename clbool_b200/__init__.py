"""clbool_b200 -- B200 (sm_100a) implementation of clBool's boolean sparse hot path.

Mirrors the reference's public surface (include/clbool.hpp): ``Controls`` /
``create_controls``, ``matrix_dcsr`` / ``matrix_coo`` / ``matrix_csr`` and the
``dcsr`` / ``coo`` / ``csr`` operation namespaces, over the C ABI of
``libclbool_b200.so`` (include/clbool_b200.h).  All compute runs in
hand-written CUDA kernels; importing fails if the library is not built.
"""
from . import coo, csr, dcsr, sizing
from ._capi import LIB_PATH, declared_symbols, lib
from .core import (ClBoolException, Controls, DeviceBuffer, create_controls, device_count, matrix_coo,
                   matrix_coo_cpu, matrix_csr, matrix_csr_cpu, matrix_dcsr, matrix_dcsr_cpu, show_devices)
from .ops import (coo_to_dcsr_shallow, csr_cpu_from_pairs, csr_from_cpu, csr_to_dcsr, dcsr_to_coo_deep,
                  dcsr_to_coo_shallow, dcsr_to_csr, fill_with, fill_with_zeroes, matrix_coo_from_gpu,
                  matrix_csr_from_gpu, matrix_dcsr_from_cpu, matrix_dcsr_from_gpu, prefix_sum)

Exception = ClBoolException  # clbool::Exception

__all__ = [
    "coo", "csr", "dcsr", "sizing", "ClBoolException", "Controls", "DeviceBuffer", "create_controls", "device_count",
    "show_devices", "matrix_coo", "matrix_coo_cpu", "matrix_csr", "matrix_csr_cpu", "matrix_dcsr",
    "matrix_dcsr_cpu", "coo_to_dcsr_shallow", "csr_cpu_from_pairs", "csr_from_cpu", "csr_to_dcsr",
    "dcsr_to_coo_deep", "dcsr_to_coo_shallow", "dcsr_to_csr", "fill_with", "fill_with_zeroes",
    "matrix_coo_from_gpu", "matrix_csr_from_gpu", "matrix_dcsr_from_cpu", "matrix_dcsr_from_gpu", "prefix_sum",
    "LIB_PATH", "lib", "declared_symbols",
]
