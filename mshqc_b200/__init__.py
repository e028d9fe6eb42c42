"""B200-native Cholesky-vector MP2 (CD-RMP2 / CD-UMP2 / CD-OMP2).

The compute lives in libmshqc_cuda.so (C ABI: include/mshqc_cd.h); this
package holds its Python binding (capi), the synthetic input recipe
(synthetic) and the build recipe (build).
"""
from . import capi  # noqa: F401

__all__ = ["capi"]
