"""clbool::coo namespace (src/coo/coo.hpp, src/coo/coo_initialization.hpp)."""
from .ops import coo_matrix_addition as matrix_addition
from .ops import sort_arrays

__all__ = ["matrix_addition", "sort_arrays"]
