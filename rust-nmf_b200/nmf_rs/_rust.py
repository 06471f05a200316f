"""Compatibility alias for code that imports the reference's native module
directly (``from nmf_rs._rust import py_nmf_run``): the same seven callables
(omicverse/rust-NMF ``rust/src/lib.rs:2177-2187``), served by the CUDA
library through :mod:`nmf_rs._native`."""
from ._native import (  # noqa: F401
    py_divergence_update_h,
    py_divergence_update_w,
    py_euclidean_update_h,
    py_euclidean_update_w,
    py_nmf_run,
    py_smoothing_matrix,
    set_num_threads,
)
