"""rustymath-b200: rustymath's dense float64 linear-algebra path on the NVIDIA B200.

`rustymath_b200.linalg` mirrors rustymath's `rm.linalg.solve`, `rm.linalg.lu` (-> `Lu`)
and `rm.matmul`; the kernels are sm_100a CUDA behind the C ABI in include/rm_cuda.h."""
from . import batched, linalg
from ._lib import NotRegular, RmError
from .batched import BatchPlan, solve_batched
from .linalg import Lu, lu, lu_solve, matmul, solve, solve_report

__all__ = ["linalg", "batched", "solve", "solve_report", "lu", "Lu", "lu_solve", "matmul", "solve_batched",
           "BatchPlan", "NotRegular", "RmError"]
