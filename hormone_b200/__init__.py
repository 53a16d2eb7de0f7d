"""hormone_b200: a B200-native implementation of HORMONE's explicit MHD step.

Host-side modules (``config``, ``grid``, ``ic``, ``binio``) are plain Python;
the step itself runs in the CUDA library ``libhormone_b200.so`` reached
through the C ABI declared in ``include/hormone_gpu.h`` (``capi``).
"""
__all__ = ["config", "grid", "ic", "binio"]
