"""clbool::csr namespace (src/csr/csr.hpp)."""
from .ops import csr_matrix_addition as matrix_addition

__all__ = ["matrix_addition"]
