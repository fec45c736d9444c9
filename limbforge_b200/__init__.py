"""B200-native implementation of the LimbForge/WolfNum batched multiprecision path.

``limbforge_b200.api`` mirrors the reference's C++ classes over the C ABI of
``liblimbforge_b200.so`` (hand-written sm_100a CUDA kernels); ``limbforge_b200.numbers``
builds and inspects arrays in the reference's element layout.  Importing ``api`` requires the
built library (``limbforge_b200.build.build()``).
"""
from . import numbers  # noqa: F401

__all__ = ["numbers"]
