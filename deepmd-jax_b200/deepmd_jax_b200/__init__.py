"""B200-native (sm_100a) Deep Potential evaluation and MD step.

Host-side mirror of deepmd-jax's model / MD interface; all device work runs
in libdpb200.so (CUDA kernels behind the C ABI in include/dpb200.h).
"""
__version__ = "0.1.0"
