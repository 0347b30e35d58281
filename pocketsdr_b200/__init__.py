"""pocketsdr_b200 - B200-native (sm_100a) signal-search and correlation hot path
of Pocket SDR behind the reference's C ABI.

Modules:
  _lib      ctypes binding of lib/libsdr_gpu.so (include/pocket_sdr_gpu.h)
  sdr_func  mirror of python/sdr_func.py's hot functions, executed on the GPU
  acquire   batched multi-signal acquisition (one plan, many PRNs x bins x sums)
  codes     spreading-code replicas and code DFTs for the acquisition plans
  synth     seeded synthetic IF generator for the benchmark configurations
  build     in-tree nvcc build of the library
"""
__version__ = "0.1.0"
