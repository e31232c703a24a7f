"""B200 (sm_100a) mean-field and time-step path of BCN-4He-DFT behind a C-ABI drop-in.

The compute lives in libhedft.so (hand-written CUDA, include/he_dft.h); this package is the
host-side mirror of the reference's call surface used by tests and the benchmark.
"""
from .config import Workload, statics_500, tddft_1000, tddft_5000_256  # noqa: F401


def Context(*a, **kw):  # noqa: N802  (constructor-style factory; loads the library lazily)
    from .context import Context as _C
    return _C(*a, **kw)
