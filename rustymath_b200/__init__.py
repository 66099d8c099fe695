"""rustymath-b200: rustymath's dense float64 linear-algebra path on the NVIDIA B200.

`rustymath_b200.linalg` mirrors rustymath's `rm.linalg.solve`, `lu` (-> `Lu`), `lu_solve`,
`det`, `slogdet`, `cholesky` and `rm.matmul`; the kernels are sm_100a CUDA behind the C ABI in
include/rm_cuda.h."""
from . import batched, linalg
from ._lib import NotPositiveDefinite, NotRegular, RmError
from .batched import BatchPlan, solve_batched
from .linalg import Lu, cholesky, det, lu, lu_inverse, lu_solve, matmul, slogdet, solve, solve_report

__all__ = ["linalg", "batched", "solve", "solve_report", "lu", "Lu", "lu_solve", "lu_inverse", "det", "slogdet",
           "cholesky", "matmul", "solve_batched", "BatchPlan", "NotRegular", "NotPositiveDefinite", "RmError"]
