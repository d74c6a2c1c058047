"""B200-native (sm_100a) physics hot path of the SolarSystemSimulator.

Modules mirror the reference's backend modules:
  selfgrav_kernel — NBodySelfGrav (all-pairs self-gravity + tracers)
The compute runs in libsss.so (include/sss.h); see build.py.
"""
from ._lib import SSSError, load as load_library  # noqa: F401

__all__ = ["SSSError", "load_library"]
