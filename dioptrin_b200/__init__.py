"""B200-native lookup-table azimuthal integration (Dioptrin's CSR path).

The CSR table is built on the GPU and integrated there by hand-written
sm_100a kernels in libdioptrin_b200.so, reached through the C ABI in
include/dioptrin_gpu.h. This package mirrors the reference's Python API:
``Integrator`` with ``integrate1d``, ``integrate2d``, ``batch1d`` and
``batch1d_iter``, and ``Cuda1dPlan`` / ``Cuda2dPlan`` from
``Integrator.prepare_cuda1d`` / ``prepare_cuda2d``.
"""
from ._native import CudaUnavailableError, RequestTimeout
from .integrator import (BatchIterator, BatchResult, Cuda1dPlan, Cuda2dPlan, Dynamic1dPlan,
                         Dynamic1dWorker, IntermediateResult1d,
                         IntegrationResult, Integrator, Poni, alloc_pinned, bslz4_compress,
                         cuda_available, is_pinned,
                         cuda_info)
from .server import RequestLoop

__all__ = ["BatchIterator", "BatchResult", "Cuda1dPlan", "Cuda2dPlan", "CudaUnavailableError",
           "Dynamic1dPlan", "Dynamic1dWorker", "IntermediateResult1d",
           "IntegrationResult", "Integrator", "Poni", "RequestLoop", "RequestTimeout",
           "alloc_pinned", "bslz4_compress", "cuda_available", "cuda_info", "is_pinned"]
