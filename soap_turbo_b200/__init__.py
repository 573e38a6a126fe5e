"""soap_turbo_b200: soap_turbo's SOAP descriptor path (get_soap, its Cartesian
derivatives and the soap_contract force VJP) on B200 GPUs.

* ``descriptor``: the reference's interface (get_soap, soap_contract,
  get_compress_indices) on host arrays, as a drop-in.
* ``context``: the same computations on device-resident neighbour lists.
* ``synthetic``: seeded synthetic structures and CSR neighbour lists.

All computation happens in libsoapb200.so (CUDA, sm_100a).
"""
from . import synthetic  # noqa: F401

__all__ = ["descriptor", "context", "synthetic"]
