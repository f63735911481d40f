"""lsms_b200: B200-native (sm_100a) tau00 multiple-scattering solve for LSMS.

The product is the CUDA library ``lsms_b200/_lib/libb200tau.so`` behind the C ABI in
``include/b200tau.h``; ``lsms_b200.tau`` is its Python host side and ``lsms_b200.workloads``
builds seeded synthetic inputs with the reference's data layouts.
"""

from . import workloads  # noqa: F401

__all__ = ["workloads", "tau", "build"]
