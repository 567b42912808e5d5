"""B200-native locate-and-link for gpu_tracking (amfaber/tracking_optimizations).

Drop-in for the reference's Python module: `batch`, `batch_file`,
`batch_rust`, `batch_file_rust`, `link_rust`, `parse_ets`.  All compute runs in libgt.so
(hand-written sm_100a CUDA kernels); there is no CPU fallback.
"""
from .gpu_tracking import batch_file_rust, batch_rust, column_names, link_rust, parse_ets
from .lib import batch, batch_file

link = link_rust

__all__ = ["batch", "batch_file", "batch_rust", "batch_file_rust", "link_rust", "link", "column_names",
           "parse_ets"]
