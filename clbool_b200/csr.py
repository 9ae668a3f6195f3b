"""clbool::csr namespace (src/csr/csr.hpp)."""
from .ops import csr_matrix_addition as matrix_addition
from .ops import csr_matrix_addition_batched as matrix_addition_batched

__all__ = ["matrix_addition", "matrix_addition_batched"]
