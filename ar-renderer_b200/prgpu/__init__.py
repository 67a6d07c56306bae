"""prgpu -- Python front end of the B200 path-tracing module.

The product is the C ABI of libprender_gpu.so (include/prgpu_api.h), a drop-in for PRender's
prender_gpu module, plus the C++ host builders of libprender_host.so (include/prhost_api.h).
This package loads both through ctypes and generates the synthetic workloads (triangle soups,
the box-and-spheres scene family) used by the tests and the benchmark.
"""

from . import abi  # noqa: F401
