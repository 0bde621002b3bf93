"""rtb200: B200-native ray traversal behind the reference's C-ABI.

The product is the shared library ``lib/libcudabvh_b200.so`` built from
``csrc/``; this package is its host-side Python mirror (ctypes binding,
seeded workload generators) used by the tests and the benchmark.
"""
from . import philox, scenes  # noqa: F401
