"""ctypes binding of ``libnmfcu.so`` (declared in ``include/nmfcu.h``).

This module is the Python side of the drop-in boundary: it exports the seven
callables of the reference's native module ``nmf_rs._rust``
(omicverse/rust-NMF ``rust/src/lib.rs:2177-2187``) with the same names,
arguments and defaults, implemented by calls into the CUDA library.  There is
no CPU fallback: if the library or a GPU is missing, the compute callables
raise ``RuntimeError``.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Optional

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("NMFCU_LIBRARY", _HERE / "libnmfcu.so"))

# Status codes (nmfcu_status).
OK, INVALID_ARG, UNSUPPORTED, OOM, CUDA, NUMERIC, TIMEOUT, NO_DEVICE, CANCELLED = range(9)

# Method ids (Algo, lib.rs:1472-1484) and stop ids (Stop, lib.rs:1507-1513).
BRUNET, LEE, OFFSET, NSNMF, HALS, EHALS, DNMF, LSNMF, SNMF_R, SNMF_L = range(10)
STOP_MAX_ITER, STOP_STATIONARY = 0, 1
PRECISIONS = {"fp64": 0, "fp32": 1, "bf16x3": 2}
MAX_RANK = 32
F64, F32 = 0, 1  # element type of a device V

(KCLASS_HSTEP, KCLASS_WSTEP, KCLASS_OBJECTIVE, KCLASS_OTHER, KCLASS_HSTEP_REFINE,
 KCLASS_WSTEP_REFINE) = range(6)
OBJECTIVE_KL, OBJECTIVE_FROBENIUS = 0, 1
NOALLOC_MAX_ROWS = 524288

_i32, _i64, _dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)


class ServerStats(ctypes.Structure):
    """Mirror of ``nmfcu_server_stats``."""

    _fields_ = [
        ("submitted", _i64), ("completed", _i64), ("failed", _i64), ("cancelled", _i64),
        ("queued", _i64), ("running", _i64), ("iterations", _i64), ("wall_ms", _dbl),
        ("p50_ms", _dbl), ("p99_ms", _dbl), ("max_ms", _dbl), ("mean_queue_ms", _dbl),
        ("budget_bytes", _i64), ("in_use_bytes", _i64), ("peak_bytes", _i64),
        ("launches", _i64), ("slots", _i32), ("peak_running", _i32),
    ]


class Options(ctypes.Structure):
    """Mirror of ``nmfcu_options``."""

    _fields_ = [
        ("method", _i32),
        ("stop", _i32),
        ("precision", _i32),
        ("rescale", _i32),
        ("max_iter", _i64),
        ("eps", _dbl),
        ("theta", _dbl),
        ("sparsity_h", _dbl),
        ("sparsity_w", _dbl),
        ("smoothness_h", _dbl),
        ("smoothness_w", _dbl),
        ("stationary_th", _dbl),
        ("check_interval", _i64),
        ("check_niter", _i64),
        ("refine_iters", _i32),
        ("device", _i32),
    ]


# Every symbol include/nmfcu.h declares, with (restype, argtypes).
SIGNATURES = {
    "nmfcu_options_default": (None, [ctypes.POINTER(Options)]),
    "nmfcu_parse_method": (_i32, [ctypes.c_char_p, ctypes.POINTER(_i32)]),
    "nmfcu_parse_stop": (_i32, [ctypes.c_char_p, ctypes.POINTER(_i32)]),
    "nmfcu_run": (_i32, [ctypes.POINTER(Options), _i64, _i64, _i64, _dp, _dp, _dp, _dp, _dp,
                         _dp, _i64, _i64p, _i64p]),
    "nmfcu_run_offset": (_i32, [ctypes.POINTER(Options), _i64, _i64, _i64, _dp, _dp, _dp, _dp,
                                _dp, _dp, _dp, _dp, _i64, _i64p, _i64p]),
    "nmfcu_run_weighted": (_i32, [ctypes.POINTER(Options), _i64, _i64, _i64, _dp, _dp, _dp, _dp,
                                  _dp, _dp, _dp, _i64, _i64p, _i64p]),
    "nmfcu_update_h_divergence": (_i32, [_i64, _i64, _i64, _dp, _dp, _dp, _dp]),
    "nmfcu_update_w_divergence": (_i32, [_i64, _i64, _i64, _dp, _dp, _dp, _dp]),
    "nmfcu_update_h_euclidean": (_i32, [_i64, _i64, _i64, _dp, _dp, _dp, _dbl, _dp]),
    "nmfcu_update_w_euclidean": (_i32, [_i64, _i64, _i64, _dp, _dp, _dp, _dbl, _dp]),
    "nmfcu_smoothing_matrix": (_i32, [_i64, _dbl, _dp]),
    "nmfcu_set_num_threads": (_i32, [_i64]),
    "nmfcu_divergence": (_i32, [_i64, _i64, _i64, _dp, _dp, _dp, _dp]),
    "nmfcu_distance": (_i32, [_i64, _i64, _i64, _dp, _dp, _dp, _dp]),
    "nmfcu_context_create": (_i32, [_i32, ctypes.POINTER(ctypes.c_void_p)]),
    "nmfcu_context_destroy": (None, [ctypes.c_void_p]),
    "nmfcu_run_device": (_i32, [ctypes.c_void_p, ctypes.POINTER(Options), _i64, _i64, _i64,
                                ctypes.c_void_p, _i32, _i64, ctypes.c_void_p, _i64,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _i64p, _i64p,
                                ctypes.c_void_p]),
    "nmfcu_run_offset_device": (_i32, [ctypes.c_void_p, ctypes.POINTER(Options), _i64, _i64,
                                       _i64, ctypes.c_void_p, _i32, _i64, ctypes.c_void_p, _i64,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, _i64p, _i64p,
                                       ctypes.c_void_p]),
    "nmfcu_consensus_stats_device": (_i32, [ctypes.c_void_p, _i64, ctypes.c_void_p, _i64,
                                            ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "nmfcu_consensus_stats_batch_device": (_i32, [ctypes.c_void_p, _i32, _i64, ctypes.c_void_p,
                                                  _i64, _i64, ctypes.POINTER(ctypes.c_double),
                                                  ctypes.POINTER(ctypes.c_double),
                                                  ctypes.c_void_p]),
    "nmfcu_shard_reduce_len": (_i64, [_i64, _i64]),
    "nmfcu_shard_create": (_i32, [ctypes.c_void_p, ctypes.POINTER(Options), _i64, _i64, _i64,
                                  ctypes.c_void_p, _i64, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]),
    "nmfcu_shard_step": (_i32, [ctypes.c_void_p, _i32, ctypes.c_void_p]),
    "nmfcu_shard_status": (_i32, [ctypes.c_void_p, _i64p, ctypes.POINTER(_i32),
                                  ctypes.c_void_p]),
    "nmfcu_shard_result": (_i32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p, _i64p, _i64p, ctypes.c_void_p]),
    "nmfcu_shard_destroy": (None, [ctypes.c_void_p]),
    "nmfcu_v_product_device": (_i32, [ctypes.c_void_p, _i32, _i64, _i64, _i64, ctypes.c_void_p,
                                      _i64, ctypes.c_void_p, _i64, ctypes.c_void_p, _i64,
                                      ctypes.c_void_p]),
    "nmfcu_context_set_timing": (_i32, [ctypes.c_void_p, _i32]),
    "nmfcu_context_kernel_time": (_i32, [ctypes.c_void_p, _i32, _i64p,
                                         ctypes.POINTER(ctypes.c_double)]),
    "nmfcu_context_reset_timing": (_i32, [ctypes.c_void_p]),
    "nmfcu_context_launch_count": (_i64, [ctypes.c_void_p]),
    "nmfcu_run_batch": (_i32, [_i32, _i32, _i64, _i64, _i64, _dp, _i32,
                               ctypes.POINTER(_i32), _dp, _dp, _dp, _dp, _i32]),
    "nmfcu_run_batch_device": (_i32, [ctypes.c_void_p, _i32, _i32, _i64, _i64, _i64,
                                      ctypes.c_void_p, _i64, _i32, ctypes.POINTER(_i32),
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "nmfcu_batch_set_shape": (_i32, [_i32]),
    "nmfcu_batch_shape_count": (_i32, []),
    "nmfcu_batch_last_shape": (_i32, []),
    "nmfcu_consensus_device": (_i32, [ctypes.c_void_p, _i64, _i32, ctypes.POINTER(_i32),
                                      ctypes.c_void_p, _i32, ctypes.POINTER(_i32),
                                      ctypes.c_void_p, ctypes.c_void_p]),
    "nmfcu_server_create": (_i32, [_i32, _i32, _i64, ctypes.POINTER(ctypes.c_void_p)]),
    "nmfcu_server_destroy": (None, [ctypes.c_void_p]),
    "nmfcu_server_submit": (_i32, [ctypes.c_void_p, ctypes.POINTER(Options), _i64, _i64, _i64,
                                   _dp, _i64, _dp, _dp, _dp, _dp, _dp, _i64, _i64p]),
    "nmfcu_server_submit_offset": (_i32, [ctypes.c_void_p, ctypes.POINTER(Options), _i64, _i64,
                                          _i64, _dp, _i64, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                          _i64, _i64p]),
    "nmfcu_server_poll": (_i32, [ctypes.c_void_p, _i64, ctypes.POINTER(_i32)]),
    "nmfcu_server_wait": (_i32, [ctypes.c_void_p, _i64, _i64, _i64p, _i64p]),
    "nmfcu_server_cancel": (_i32, [ctypes.c_void_p, _i64]),
    "nmfcu_server_get_stats": (_i32, [ctypes.c_void_p, ctypes.POINTER(ServerStats)]),
    "nmfcu_server_reset_stats": (_i32, [ctypes.c_void_p]),
    "nmfcu_run_csr": (_i32, [ctypes.POINTER(Options), _i64, _i64, _i64, _i64, _i64p,
                             ctypes.POINTER(_i32), _dp, _dp, _dp, _dp, _dp, _dp, _i64, _i64p,
                             _i64p]),
    "nmfcu_run_csr_device": (_i32, [ctypes.c_void_p, ctypes.POINTER(Options), _i64, _i64, _i64,
                                    _i64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _i64p,
                                    _i64p, ctypes.c_void_p]),
    "nmfcu_objective_noalloc": (_i32, [_i32, _i64, _i64, _i64, ctypes.c_void_p, _i64,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]),
    "nmfcu_last_error": (ctypes.c_char_p, []),
    "nmfcu_status_string": (ctypes.c_char_p, [_i32]),
    "nmfcu_abi_version": (_i32, []),
    "nmfcu_device_count": (_i32, []),
}

_lib = None


def load():
    """Load libnmfcu.so and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"CUDA backend not available: {LIB_PATH} is missing. Build it with "
            "`make -C rust-nmf_b200/csrc` (or __graft_entry__.build())."
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def available() -> bool:
    try:
        load()
        return True
    except (RuntimeError, OSError):
        return False


def device_count() -> int:
    return int(load().nmfcu_device_count())


def check(status: int) -> None:
    """Raise the Python exception the reference's contract implies."""
    if status == OK:
        return
    msg = load().nmfcu_last_error().decode(errors="replace")
    if status == INVALID_ARG:
        raise ValueError(msg)
    if status == UNSUPPORTED:
        raise NotImplementedError(msg)
    if status == OOM:
        raise MemoryError(msg)
    if status == CANCELLED:
        import concurrent.futures

        raise concurrent.futures.CancelledError(msg)
    raise RuntimeError(f"nmfcu: {load().nmfcu_status_string(status).decode()}: {msg}")


def _f64(a, name: str) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if arr.ndim != 2:
        raise ValueError(f"{name} must be 2-D, got shape {arr.shape}")
    return arr


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def parse_method(name: str) -> int:
    out = _i32(0)
    check(load().nmfcu_parse_method(str(name).encode(), ctypes.byref(out)))
    return int(out.value)


def parse_stop(name: str) -> int:
    out = _i32(0)
    check(load().nmfcu_parse_stop(str(name).encode(), ctypes.byref(out)))
    return int(out.value)


def default_options() -> Options:
    o = Options()
    load().nmfcu_options_default(ctypes.byref(o))
    return o


def _shapes_of(vshape: tuple, w: np.ndarray, h: np.ndarray) -> tuple[int, int, int]:
    n, p = vshape
    r = w.shape[1]
    if w.shape[0] != n or h.shape != (r, p):
        raise ValueError(
            f"shape mismatch: V {tuple(vshape)}, W {w.shape}, H {h.shape} "
            "(need n x r and r x p)")
    return int(n), int(p), int(r)


def _shapes(v: np.ndarray, w: np.ndarray, h: np.ndarray) -> tuple[int, int, int]:
    return _shapes_of(v.shape, w, h)


# ---------------------------------------------------------------------------
# The seven callables of nmf_rs._rust
# ---------------------------------------------------------------------------

def set_num_threads(n: int) -> bool:
    """set_num_threads (lib.rs:1841-1847).  No CPU pool exists: returns False."""
    return bool(load().nmfcu_set_num_threads(int(n)))


def py_divergence_update_h(v, w, h) -> np.ndarray:
    """One brunet H update (lib.rs:1851-1862)."""
    v, w, h = _f64(v, "V"), _f64(w, "W"), _f64(h, "H")
    n, p, r = _shapes(v, w, h)
    out = np.empty((r, p), dtype=np.float64)
    check(load().nmfcu_update_h_divergence(n, p, r, _ptr(v), _ptr(w), _ptr(h), _ptr(out)))
    return out


def py_divergence_update_w(v, w, h) -> np.ndarray:
    """One brunet W update (lib.rs:1866-1877)."""
    v, w, h = _f64(v, "V"), _f64(w, "W"), _f64(h, "H")
    n, p, r = _shapes(v, w, h)
    out = np.empty((n, r), dtype=np.float64)
    check(load().nmfcu_update_w_divergence(n, p, r, _ptr(v), _ptr(w), _ptr(h), _ptr(out)))
    return out


def py_euclidean_update_h(v, w, h, eps) -> np.ndarray:
    """One lee H update (lib.rs:1880-1892)."""
    v, w, h = _f64(v, "V"), _f64(w, "W"), _f64(h, "H")
    n, p, r = _shapes(v, w, h)
    out = np.empty((r, p), dtype=np.float64)
    check(load().nmfcu_update_h_euclidean(n, p, r, _ptr(v), _ptr(w), _ptr(h), float(eps),
                                          _ptr(out)))
    return out


def py_euclidean_update_w(v, w, h, eps) -> np.ndarray:
    """One lee W update (lib.rs:1895-1907)."""
    v, w, h = _f64(v, "V"), _f64(w, "W"), _f64(h, "H")
    n, p, r = _shapes(v, w, h)
    out = np.empty((n, r), dtype=np.float64)
    check(load().nmfcu_update_w_euclidean(n, p, r, _ptr(v), _ptr(w), _ptr(h), float(eps),
                                          _ptr(out)))
    return out


def py_smoothing_matrix(r: int, theta: float) -> np.ndarray:
    """nsNMF smoothing matrix (lib.rs:2172-2175)."""
    r = int(r)
    out = np.empty((r, r), dtype=np.float64)
    check(load().nmfcu_smoothing_matrix(r, float(theta), _ptr(out) if r else None))
    return out


def py_nmf_run(algo: str, v, w0, h0, max_iter: int, *, eps: float = 1e-9,
               rescale: bool = True, theta: float = 0.5, offset=None, weight=None,
               sparsity_h: float = 0.0, sparsity_w: float = 0.0, smoothness_h: float = 0.0,
               smoothness_w: float = 0.0, stop: str = "max_iter",
               stationary_th: float = 2.220446049250313e-16, check_interval: int = 50,
               check_niter: int = 10, num_threads: Optional[int] = None,
               precision: str = "fp64", refine_iters: int = 2, device: int = 0) -> dict:
    """The full loop (lib.rs:1934-2169).  Same positional / keyword signature
    and defaults; ``precision``, ``refine_iters`` and ``device`` are engine
    extensions.  ``num_threads`` is accepted and ignored (there is no CPU
    thread pool).  Returns ``{"W", "H", "n_iter", "deviances"}``, plus
    ``"offset"`` for the offset method (lib.rs:2161-2165)."""
    o, v, w0, h0, n, p, r = build_run_options(
        algo, v, w0, h0, max_iter, eps=eps, rescale=rescale, theta=theta, offset=offset,
        weight=weight, sparsity_h=sparsity_h, sparsity_w=sparsity_w, smoothness_h=smoothness_h,
        smoothness_w=smoothness_w, stop=stop, stationary_th=stationary_th,
        check_interval=check_interval, check_niter=check_niter, num_threads=num_threads,
        precision=precision, refine_iters=refine_iters, device=device)
    W = np.empty((n, r), dtype=np.float64)
    H = np.empty((r, p), dtype=np.float64)
    cap = o.max_iter + 1
    dev = np.empty(cap, dtype=np.float64)
    nd, ni = _i64(0), _i64(0)
    if o.method == OFFSET:
        off0 = None
        if offset is not None:
            off0 = np.ascontiguousarray(np.asarray(offset, dtype=np.float64))
            if off0.shape != (n,):
                raise ValueError(f"offset.shape {off0.shape} != ({n},)")
        off = np.empty(n, dtype=np.float64)
        check(load().nmfcu_run_offset(
            ctypes.byref(o), n, p, r, _ptr(v), _ptr(w0), _ptr(h0),
            _ptr(off0) if off0 is not None else None, _ptr(W), _ptr(H), _ptr(off), _ptr(dev),
            cap, ctypes.byref(nd), ctypes.byref(ni)))
        return {"W": W, "H": H, "offset": off, "n_iter": int(ni.value),
                "deviances": list(dev[: nd.value])}
    if o.method == LSNMF:
        S = np.ascontiguousarray(np.asarray(weight, dtype=np.float64))
        if S.shape != v.shape:
            raise ValueError(f"weight.shape {S.shape} != V.shape {v.shape}")
        check(load().nmfcu_run_weighted(
            ctypes.byref(o), n, p, r, _ptr(v), _ptr(S), _ptr(w0), _ptr(h0), _ptr(W), _ptr(H),
            _ptr(dev), cap, ctypes.byref(nd), ctypes.byref(ni)))
        return {"W": W, "H": H, "n_iter": int(ni.value), "deviances": list(dev[: nd.value])}
    check(load().nmfcu_run(ctypes.byref(o), n, p, r, _ptr(v), _ptr(w0), _ptr(h0), _ptr(W),
                           _ptr(H), _ptr(dev), cap, ctypes.byref(nd), ctypes.byref(ni)))
    return {"W": W, "H": H, "n_iter": int(ni.value), "deviances": list(dev[: nd.value])}


def csr_arrays(V):
    """(indptr int64, indices int32, data f64, (n, p)) of a scipy sparse V in
    canonical CSR form (duplicates summed, indices sorted), C-contiguous."""
    import scipy.sparse as sp

    m = sp.csr_matrix(V, dtype=np.float64, copy=True)
    m.sum_duplicates()
    m.sort_indices()
    if m.nnz > np.iinfo(np.int32).max:
        raise NotImplementedError("a sparse V holds at most 2^31 - 1 stored entries")
    return (np.ascontiguousarray(m.indptr, dtype=np.int64),
            np.ascontiguousarray(m.indices, dtype=np.int32),
            np.ascontiguousarray(m.data, dtype=np.float64), m.shape)


def py_nmf_run_csr(algo: str, v, w0, h0, max_iter: int, **kw) -> dict:
    """py_nmf_run for a sparse V (scipy.sparse, any format): the loop over its
    stored entries (nmfcu_run_csr), lee / brunet / hals / dnmf in FP64.  Same
    keywords and result as :func:`py_nmf_run`; the reference densifies V
    instead (python/nmf_rs/__init__.py:495)."""
    indptr, indices, data, (n, p) = csr_arrays(v)
    o, _, w0, h0, n, p, r = build_run_options(algo, None, w0, h0, max_iter, shape=(n, p), **kw)
    W = np.empty((n, r), dtype=np.float64)
    H = np.empty((r, p), dtype=np.float64)
    cap = o.max_iter + 1
    dev = np.empty(cap, dtype=np.float64)
    nd, ni = _i64(0), _i64(0)
    check(load().nmfcu_run_csr(
        ctypes.byref(o), n, p, r, int(data.size),
        indptr.ctypes.data_as(_i64p), indices.ctypes.data_as(ctypes.POINTER(_i32)), _ptr(data),
        _ptr(w0), _ptr(h0), _ptr(W), _ptr(H), _ptr(dev), cap, ctypes.byref(nd), ctypes.byref(ni)))
    return {"W": W, "H": H, "n_iter": int(ni.value), "deviances": list(dev[: nd.value])}


def build_run_options(algo: str, v, w0, h0, max_iter: int, *, eps: float = 1e-9,
                      rescale: bool = True, theta: float = 0.5, offset=None, weight=None,
                      sparsity_h: float = 0.0, sparsity_w: float = 0.0,
                      smoothness_h: float = 0.0, smoothness_w: float = 0.0,
                      stop: str = "max_iter", stationary_th: float = 2.220446049250313e-16,
                      check_interval: int = 50, check_niter: int = 10,
                      num_threads: Optional[int] = None, precision: str = "fp64",
                      refine_iters: int = 2, device: int = 0, shape=None):
    """py_nmf_run's argument handling (lib.rs:1934-1971): the checks in the
    reference's order and the ``nmfcu_options`` they produce.  Returns
    ``(options, V, W0, H0, n, p, r)`` with the arrays as C-contiguous f64.
    With ``shape=(n, p)`` V is not given (a sparse V) and None is returned
    in its place."""
    o = default_options()
    o.method = parse_method(algo)            # Algo::from_str, lib.rs:1956
    o.stop = parse_stop(stop)                # Stop::from_str, lib.rs:1957
    if o.method == LSNMF and weight is None:  # lib.rs:1967-1971
        raise ValueError("method='lsnmf' requires a `weight` matrix of the same shape as V")
    if num_threads is not None and int(num_threads) < 0:
        raise OverflowError("num_threads must be a non-negative integer")
    w0, h0 = _f64(w0, "W0"), _f64(h0, "H0")
    if shape is None:
        v = _f64(v, "V")
        n, p, r = _shapes(v, w0, h0)
    else:
        n, p, r = _shapes_of(tuple(shape), w0, h0)
    try:
        o.precision = PRECISIONS[str(precision).lower()]
    except KeyError:
        raise ValueError(f"unknown precision {precision!r}: supported fp64, fp32, bf16x3") from None
    o.max_iter = int(max_iter)
    if o.max_iter < 0:
        raise OverflowError("max_iter must be a non-negative integer")
    o.eps = float(eps)
    o.rescale = int(bool(rescale))
    o.theta = float(theta)
    o.sparsity_h, o.sparsity_w = float(sparsity_h), float(sparsity_w)
    o.smoothness_h, o.smoothness_w = float(smoothness_h), float(smoothness_w)
    o.stationary_th = float(stationary_th)
    o.check_interval = int(check_interval)
    o.check_niter = int(check_niter)
    o.refine_iters = int(refine_iters)
    o.device = int(device)
    return o, v, w0, h0, n, p, r


def divergence(v, w, h) -> float:
    """kl_divergence(V, WH) on the GPU (lib.rs:1410-1431)."""
    v, w, h = _f64(v, "V"), _f64(w, "W"), _f64(h, "H")
    n, p, r = _shapes(v, w, h)
    out = ctypes.c_double(0.0)
    check(load().nmfcu_divergence(n, p, r, _ptr(v), _ptr(w), _ptr(h), ctypes.byref(out)))
    return float(out.value)


def distance(v, w, h) -> float:
    """euclidean_distance(V, WH) = 0.5 ||V - WH||^2 on the GPU (lib.rs:1434-1445)."""
    v, w, h = _f64(v, "V"), _f64(w, "W"), _f64(h, "H")
    n, p, r = _shapes(v, w, h)
    out = ctypes.c_double(0.0)
    check(load().nmfcu_distance(n, p, r, _ptr(v), _ptr(w), _ptr(h), ctypes.byref(out)))
    return float(out.value)


# ---------------------------------------------------------------------------
# Device-resident runs (inputs already in HBM; used by the benchmark and by
# callers that keep V on the GPU, e.g. as a torch tensor).
# ---------------------------------------------------------------------------

class Context:
    """An ``nmfcu_context``: device scratch reused across device-pointer runs."""

    def __init__(self, device: int = 0):
        self._lib = load()
        h = ctypes.c_void_p()
        check(self._lib.nmfcu_context_create(int(device), ctypes.byref(h)))
        self.handle = h
        self.device = int(device)

    def close(self):
        if getattr(self, "handle", None):
            self._lib.nmfcu_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, opts: Options, n: int, p: int, r: int, v_ptr: int, v_dtype: int, ldv: int,
            w_ptr: int, h_ptr: int, *, v64_ptr: int = 0, ldv64: int = 0, dev_ptr: int = 0,
            stream: int = 0) -> tuple[int, int]:
        nd, ni = _i64(0), _i64(0)
        check(self._lib.nmfcu_run_device(
            self.handle, ctypes.byref(opts), n, p, r, ctypes.c_void_p(v_ptr), v_dtype, ldv,
            ctypes.c_void_p(v64_ptr or None), ldv64, ctypes.c_void_p(w_ptr),
            ctypes.c_void_p(h_ptr), ctypes.c_void_p(dev_ptr or None), ctypes.byref(nd),
            ctypes.byref(ni), ctypes.c_void_p(stream or None)))
        return int(ni.value), int(nd.value)

    def v_product(self, trans: int, n: int, p: int, l: int, v_ptr: int, ldv: int, x_ptr: int,
                  ldx: int, out_ptr: int, ldo: int, stream: int = 0):
        """out = V X (trans 0) or V^T X (trans 1) on device pointers."""
        check(self._lib.nmfcu_v_product_device(
            self.handle, int(trans), n, p, l, ctypes.c_void_p(v_ptr), ldv, ctypes.c_void_p(x_ptr),
            ldx, ctypes.c_void_p(out_ptr), ldo, ctypes.c_void_p(stream or None)))

    def set_timing(self, on: bool):
        check(self._lib.nmfcu_context_set_timing(self.handle, int(bool(on))))

    def reset_timing(self):
        check(self._lib.nmfcu_context_reset_timing(self.handle))

    def kernel_time(self, kclass: int) -> tuple[int, float]:
        n = _i64(0)
        ms = ctypes.c_double(0.0)
        check(self._lib.nmfcu_context_kernel_time(self.handle, int(kclass), ctypes.byref(n),
                                                  ctypes.byref(ms)))
        return int(n.value), float(ms.value)

    def launch_count(self) -> int:
        return int(self._lib.nmfcu_context_launch_count(self.handle))
