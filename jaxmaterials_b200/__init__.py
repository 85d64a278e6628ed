"""B200-native Moulinec-Suquet Lippmann-Schwinger solver (drop-in for the
yang-chen-2022/JaxMaterials solver path).

The compute runs in ``liblippmannschwinger.so`` (hand-written sm_100a CUDA behind a
C ABI, declared in ``include/lippmann_schwinger.h``); this package is the Python
binding. There is no CPU fallback: every entry point raises if the library is missing.
"""

from .common import GridSpec  # noqa: F401

__all__ = ["GridSpec"]
