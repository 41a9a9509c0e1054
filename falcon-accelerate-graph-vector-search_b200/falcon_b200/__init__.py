"""falcon_b200: B200-native graph vector search (Falcon's traversal path).

The search runs in libfalcon_b200.so (hand-written sm_100a kernels behind the
C ABI in include/falcon.h); this package is the host-side mirror of the
reference's host interface plus data preparation helpers.
"""
from .formats import Graph, read_fpga_index, write_fpga_index
from .index import FalconIndex, make_params, vadd

__all__ = ["FalconIndex", "Graph", "make_params", "vadd", "read_fpga_index", "write_fpga_index"]
