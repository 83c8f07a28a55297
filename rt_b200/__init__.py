"""rt_b200: B200-native ray-tracing engine for spectrograph schemes.

The compute lives in librtb200.so (hand-written sm_100a CUDA behind the C ABI
of include/rtb.h); this package holds the ctypes binding (ffi), the
benchmark schemes (schemes) and the host-side driver (engine).
"""
