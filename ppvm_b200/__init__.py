"""ppvm_b200 — a B200-native engine for the Heisenberg-picture PauliSum path of ppvm.

``PauliSum`` mirrors ``ppvm.PauliSum`` (ppvm-python/src/ppvm/paulisum.py in the
reference) and drives the CUDA library ``libppvm_cuda.so`` through its C ABI
(include/ppvm_cuda.h).  Importing the package does not touch the GPU; the library is
loaded on first use and a missing or unloadable library raises immediately.
"""

__all__ = ["PauliSum", "LossyPauliSum", "gates", "circuits"]


def __getattr__(name):
    if name in ("PauliSum", "LossyPauliSum"):
        from . import paulisum

        return getattr(paulisum, name)
    if name in ("gates", "circuits"):
        import importlib

        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
