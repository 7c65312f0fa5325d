"""B200-native (sm_100a) H2 matrix apply engine behind H2Pack's H2P_matvec / H2P_matmul."""
from ._abi import (KRNL_COULOMB, KRNL_GAUSSIAN, KRNL_MATERN32, KRNL_RPY, PREC_FP64, PREC_MIXED,
                   ROW_MAJOR, COL_MAJOR, libh2gpu, libh2pack_gpu)
from .h2pack import H2Matrix, Image, direct_sum, plan_check
from .h2file import H2File, read_h2, write_h2

__all__ = ["H2Matrix", "Image", "direct_sum", "plan_check", "H2File", "read_h2", "write_h2", "libh2gpu", "libh2pack_gpu", "KRNL_COULOMB", "KRNL_GAUSSIAN",
           "KRNL_MATERN32", "KRNL_RPY", "PREC_FP64", "PREC_MIXED", "ROW_MAJOR", "COL_MAJOR"]
