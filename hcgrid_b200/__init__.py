"""B200-native convolution gridder (drop-in for HCGrid's gridding path).

The product is the native library built from hcgrid_b200/csrc (C ABI in
include/hcgrid_c.h); this package holds its build step, a ctypes binding
(`api`) and the seeded workload generator (`synth`).
"""
from . import api  # noqa: F401
from .api import Context, Field, Target, HcgError  # noqa: F401
