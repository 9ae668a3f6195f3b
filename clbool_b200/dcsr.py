"""clbool::dcsr namespace (src/dcsr/dcsr.hpp)."""
from .ops import kronecker_product, matrix_multiplication, matrix_multiplication_hash, transpose, workload

__all__ = ["matrix_multiplication_hash", "matrix_multiplication", "kronecker_product", "transpose", "workload"]
