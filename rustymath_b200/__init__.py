"""rustymath-b200: rustymath's dense float64 linear-algebra path on the NVIDIA B200.

`rustymath_b200.linalg` mirrors rustymath's `rm.linalg.solve`, `rm.linalg.lu` (-> `Lu`)
and `rm.matmul`; the kernels are sm_100a CUDA behind the C ABI in include/rm_cuda.h."""
from . import linalg
from ._lib import NotRegular, RmError
from .linalg import Lu, lu, lu_solve, matmul, solve, solve_report

__all__ = ["linalg", "solve", "solve_report", "lu", "Lu", "lu_solve", "matmul", "NotRegular", "RmError"]
