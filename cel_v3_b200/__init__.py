"""B200-native implementation of the CEL (hpcdkhab/cel_v3) solver hot path.

The compute path is libcelgpu.so (hand-written sm_100a CUDA behind the C ABI
in include/celgpu.h); `cel_v3_b200.celgpu` is its ctypes binding and
`cel_v3_b200.synth` builds the seeded synthetic workloads.  The binding is
imported lazily so that the CPU-only parts (synthetic inputs, build) work on
machines without the library.
"""
import importlib

__all__ = ["celgpu", "synth", "build"]


def __getattr__(name):
    if name in __all__:
        return importlib.import_module(f"{__name__}.{name}")
    raise AttributeError(name)
