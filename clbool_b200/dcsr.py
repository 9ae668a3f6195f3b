"""clbool::dcsr namespace (src/dcsr/dcsr.hpp), plus the learned single-pass form."""
from .ops import (kronecker_product, matrix_multiplication, matrix_multiplication_hash, reduce, submatrix, transpose,
                  workload)
from .sizing import RowSizer, matrix_multiplication_learned, row_features, row_nnz
from .batched import (autotune, matrix_multiplication_batched, matrix_multiplication_batched_learned,
                      matrix_multiplication_tuned, matrix_union, tuning)

__all__ = ["matrix_multiplication_hash", "matrix_multiplication", "kronecker_product", "transpose", "workload",
           "submatrix", "reduce",
           "matrix_multiplication_learned", "RowSizer", "row_features", "row_nnz", "matrix_multiplication_batched",
           "matrix_multiplication_batched_learned", "matrix_multiplication_tuned", "matrix_union", "autotune", "tuning"]
