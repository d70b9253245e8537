"""rpp_b200 — B200-native drop-in for RPP's batched audio tensor path (rppt_* audio entry points).

The product is the C-ABI library rpp_b200/librppb.so (headers in include/); this package holds its
sources (csrc/), the nvcc build (build.py), a ctypes binding (lib.py), a Python mirror of the
reference's audio interface (audio.py), ABI types (types.py) and seeded synthetic workloads
(synth.py).
"""
from . import types  # noqa: F401
