"""galoisgpu_b200 -- B200 (sm_100a) frontier-traversal engine for the
data-driven worklist BFS and SSSP path of LonestarGPU v3, with connected
components (apps/cc), PageRank (apps/pr) and maximal independent set
(apps/mis) on the same engine.

The compute lives in libgft.so (hand-written CUDA for sm_100a behind the C
ABI of include/gft.h); this package is the Python host side.
"""

from .graph import (  # noqa: F401
    Batch,
    DEFAULT_DELTA,
    GFT_NO_PARENT,
    INF,
    CSRGraph,
    DeviceGraph,
    Engine,
    Tune,
    output,
    output_gz,
    reach_stats,
    read_node_data,
    write_node_data,
    write_cc_output,
    write_pr_output,
    write_mis_output,
)
from ._lib import GftError, load  # noqa: F401

__version__ = "0.1.0"
