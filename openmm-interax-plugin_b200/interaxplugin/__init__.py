"""interaxplugin: the InteraxFF short-range path on B200 GPUs.

The Force classes mirror the reference plugin's API (same class names, method names, defaults and errors); a
Context evaluates them with the hand-written sm_100a CUDA kernels of libinterax_b200.so through its C ABI
(include/interax_b200.h).  There is no CPU fallback: creating a Context fails loudly when the library or a GPU is
missing.
"""
from .forces import (OpenMMException, Force, InteraxPairForce, InteraxDispersionForce, InteraxExchangeForce,
                     InteraxShortRangeForce, InteraxThreeBodyForce, System, computeC9)

__all__ = ["OpenMMException", "Force", "InteraxPairForce", "InteraxDispersionForce", "InteraxExchangeForce",
           "InteraxShortRangeForce", "InteraxThreeBodyForce", "System", "computeC9"]


def __getattr__(name):
    # The Context pulls in the C-ABI binding; import it lazily so that the Force classes work without a GPU.
    if name in ("Context", "State", "Platform"):
        from . import context
        return getattr(context, name)
    if name == "BatchContext":
        from . import batch
        return batch.BatchContext
    if name == "Server":
        from . import server
        return server.Server
    if name in ("XmlSerializer",):
        from . import serialization
        return getattr(serialization, name)
    raise AttributeError(name)
