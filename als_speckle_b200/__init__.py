"""B200-native phase retrieval with the speckle.phasing API (dhparks/als_speckle).

Submodules load on first use, so ``python -m als_speckle_b200.build`` works
before the library exists.
"""
import importlib

__all__ = ["phasing", "engine", "masking", "io", "gpu", "synth", "serving", "distributed", "workloads"]


def __getattr__(name):
    if name in __all__:
        return importlib.import_module("." + name, __name__)
    raise AttributeError(name)
