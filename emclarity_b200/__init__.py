"""emclarity_b200 -- B200-native (sm_100a) orientation-search hot path of emClarity.

The compute lives in libemc_b200.so (hand-written CUDA behind the C-ABI in
include/emc_b200.h); this package is the Python mirror of the reference's operator
interface (interpolator / fourierTransformer / mexCTF / mexSF3D / the search loop).
"""
from ._lib import EmcError, load  # noqa: F401

__all__ = ["EmcError", "load", "api", "synthetic"]


def __getattr__(name):
    # api / synthetic import torch; load them lazily so that the C-ABI binding alone
    # (used by CPU-only checks) does not pay for it.
    if name in ("api", "synthetic"):
        import importlib
        return importlib.import_module("." + name, __name__)
    raise AttributeError(name)
