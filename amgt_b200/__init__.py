"""amgt_b200: B200 (sm_100a) mBSR SpGEMM / SpMV behind HYPRE's AmgT hooks.

The kernels live in libamgt_b200.so (CUDA, built in-tree by
``python amgt_b200/build.py``); this package is the Python face of its C ABI
(include/amgt_b200.h).  Importing it loads the library and fails loudly
when it is missing.
"""
from ._lib import BF16, DOUBLE, FLOAT, HALF, AmgtError, lib  # noqa: F401
from .mbsr import (Bsr, CsrOwned, init, kernel_launch_count, precision_for_level,  # noqa: F401
                   set_level_policy, spgemm)
from .hypre import (CSRMatrix, hypre_CSRMatrixMatvecCusparseNewAPI,  # noqa: F401
                    hypre_Level, hypreDevice_CSRSpGemm)

lib()
