"""spsim_b200: spsim's structure-factor and detector-chain path on B200 (sm_100a).

Layers:
  include/spsim_b200.h, include/spsim.h   the C ABI of libspsim_b200.so
  spsim_b200.core                          Python API on torch device tensors
  spsim_b200.spsim / spsim_pybackend      drop-in for spsim's Python module
  spsim_b200.autograd                      torch.autograd.Function with the adjoint kernel
  spsim_b200.dist                          sharding over ranks (torch.distributed)
The library is built in-tree by `python -m spsim_b200.build`.
"""
from ._native import PREC_F32, PREC_F32_FAST, PREC_FP64, SpsimError, device_count, version  # noqa: F401

__version__ = "0.1.0"
