"""Consensus clustering over many NMF restarts and ranks.

The reference drives this workflow as a serial Python loop of ``nmf()``
calls followed by numpy/scipy metrics (omicverse/rust-NMF
``examples/build_scaling_notebook.py:121-208``): for each rank k, n_runs
restarts from ``default_rng(2024 + run)`` with W0, H0 ~ U(0, sqrt(mean(V)/k));
each run's columns are clustered by argmax over H; the consensus matrix is
the mean of the runs' connectivity matrices; the cophenetic correlation
(average linkage on 1 - consensus) and the dispersion coefficient summarise
it.

Here all restarts of all ranks run as one batch on the GPU
(``nmfcu_run_batch_device``: stacked factors, every V tile shared by a
group of solves, CUDA-graph iteration blocks), and the consensus matrices
are built on the GPU (``nmfcu_consensus_device``).  ``batched=False`` runs
the same solves one by one through the single-solve engine, for comparison.
"""
from __future__ import annotations

import ctypes
import time
from typing import Iterable

import numpy as np

from . import _native

__all__ = [
    "restart_starts",
    "run_batch",
    "consensus_sweep",
    "connectivity_matrix",
    "cophenetic_correlation",
    "dispersion_coefficient",
    "consensus_stats",
    "consensus_stats_batch",
]


# ---------------------------------------------------------------------------
# The reference's metrics (examples/build_scaling_notebook.py:121-141)
# ---------------------------------------------------------------------------

def connectivity_matrix(H: np.ndarray) -> np.ndarray:
    """1 where two columns share their argmax component, else 0."""
    cluster = np.argmax(H, axis=0)
    return (cluster[:, None] == cluster[None, :]).astype(np.float64)


def cophenetic_correlation(consensus: np.ndarray) -> float:
    """Correlation between 1 - C and the cophenetic distances of an
    average-linkage tree built on 1 - C (Brunet et al. 2004), on the host
    with scipy; 1 when either has no spread.

    The notebook helper this follows (build_scaling_notebook.py:126-137)
    takes element 0 of ``cophenet(Z, cond)`` -- the coefficient itself --
    as the cophenetic distances and then returns 1.0 because a scalar has no
    spread, so it reports 1.0 for every matrix; this returns the
    coefficient.  ``consensus_stats`` computes the same on the GPU."""
    from scipy.cluster.hierarchy import cophenet, linkage
    from scipy.spatial.distance import squareform

    c = np.array(consensus, dtype=np.float64, copy=True)
    np.fill_diagonal(c, 1.0)
    cond = squareform(1.0 - c, checks=False)
    if cond.size < 2 or cond.std() == 0:
        return 1.0
    coef, coph = cophenet(linkage(cond, method="average"), cond)
    if coph.std() == 0:
        return 1.0
    return float(coef)


def consensus_stats(C, ctx=None) -> tuple[float, float]:
    """(cophenetic correlation, dispersion coefficient) of a consensus
    matrix held on the GPU (f32 torch tensor, p x p, unit column stride),
    computed there (``nmfcu_consensus_stats_device``: average linkage by the
    nearest-neighbour chain, the same tree as scipy's)."""
    import torch

    if C.device.type != "cuda" or C.dtype != torch.float32 or C.stride(1) != 1:
        raise ValueError("C must be an f32 CUDA tensor with unit column stride")
    own = ctx is None
    ctx = ctx or _native.Context(C.device.index or 0)
    coph, disp = ctypes.c_double(0.0), ctypes.c_double(0.0)
    try:
        _native.check(_native.load().nmfcu_consensus_stats_device(
            ctx.handle, C.shape[0], ctypes.c_void_p(C.data_ptr()), C.stride(0),
            ctypes.byref(coph), ctypes.byref(disp),
            ctypes.c_void_p(torch.cuda.current_stream(C.device).cuda_stream)))
    finally:
        if own:
            ctx.close()
    return float(coph.value), float(disp.value)


def consensus_stats_batch(C, ctx=None) -> list[tuple[float, float]]:
    """``consensus_stats`` of every matrix of a stacked (count x p x p) f32
    device tensor, with the average-linkage trees of all of them built
    concurrently (``nmfcu_consensus_stats_batch_device``)."""
    count, p, p2 = C.shape
    if p != p2:
        raise ValueError(f"consensus matrices must be square, got {tuple(C.shape)}")
    C = C.contiguous()
    own = ctx is None
    if own:
        ctx = _native.Context(C.device.index or 0)
    coph = (ctypes.c_double * count)()
    disp = (ctypes.c_double * count)()
    try:
        import torch

        _native.check(_native.load().nmfcu_consensus_stats_batch_device(
            ctx.handle, count, p, ctypes.c_void_p(C.data_ptr()), p, p * p, coph, disp,
            ctypes.c_void_p(torch.cuda.current_stream(C.device).cuda_stream)))
    finally:
        if own:
            ctx.close()
    return [(float(coph[m]), float(disp[m])) for m in range(count)]


def dispersion_coefficient(consensus: np.ndarray) -> float:
    """Kim & Park 2007: mean of 4 (C - 0.5)^2; 1 means perfectly stable."""
    c = np.asarray(consensus, dtype=np.float64)
    return float((4.0 * (c - 0.5) ** 2).mean())


# ---------------------------------------------------------------------------
# Starting points and the batched solve
# ---------------------------------------------------------------------------

def restart_starts(V: np.ndarray, rank: int, n_runs: int, base_seed: int = 2024):
    """The reference's restart starting points: run r draws W0 (n x rank)
    then H0 (rank x p) from default_rng(base_seed + r), U(0, sqrt(mean V / rank))."""
    n, p = V.shape
    scale = float(np.sqrt(V.mean() / rank))
    out = []
    for run in range(n_runs):
        gen = np.random.default_rng(base_seed + run)
        W0 = gen.uniform(0, scale, (n, rank))
        H0 = gen.uniform(0, scale, (rank, p))
        out.append((W0, H0))
    return out


def _stack(starts):
    ranks = np.array([w.shape[1] for w, _ in starts], dtype=np.int32)
    W = np.ascontiguousarray(np.concatenate([w for w, _ in starts], axis=1), dtype=np.float64)
    H = np.ascontiguousarray(np.concatenate([h for _, h in starts], axis=0), dtype=np.float64)
    return ranks, W, H


def _unstack(ranks, W, H):
    out, off = [], 0
    for r in ranks:
        out.append((W[:, off:off + r].copy(), H[off:off + r].copy()))
        off += int(r)
    return out


def _ranks_ptr(ranks: np.ndarray):
    return ranks.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def set_batch_shape(shape="auto") -> None:
    """Shape of the batched kernel (solves a CTA carries, CTAs resident per
    multiprocessor): ``"auto"`` -- the default -- times the candidate shapes on
    the first batched run of each problem (device, precision, n, p, ranks;
    runs of 20 or more iterations) and keeps the fastest; an int in
    ``range(batch_shape_count())`` forces one.  Every shape gives the same
    results.  Process-wide."""
    lib = _native.load()
    code = -1 if shape == "auto" else int(shape)
    _native.check(lib.nmfcu_batch_set_shape(code))


def batch_shape_count() -> int:
    return int(_native.load().nmfcu_batch_shape_count())


def last_batch_shape() -> int:
    """The shape the last batched run used (-1 before the first)."""
    return int(_native.load().nmfcu_batch_last_shape())


def run_batch(V: np.ndarray, starts, max_iter: int, *, method: str = "brunet",
              precision: str = "fp64", device: int = 0):
    """Run every (W0, H0) in ``starts`` on V as one batch and return a list
    of (W, H): host arrays in, host arrays out (``nmfcu_run_batch``)."""
    V = np.ascontiguousarray(np.asarray(V, dtype=np.float64))
    ranks, W0, H0 = _stack(starts)
    W = np.empty_like(W0)
    H = np.empty_like(H0)
    lib = _native.load()
    n, p = V.shape
    _native.check(lib.nmfcu_run_batch(
        _native.parse_method(method), _native.PRECISIONS[precision], int(max_iter), n, p,
        _native._ptr(V), len(ranks), _ranks_ptr(ranks), _native._ptr(W0), _native._ptr(H0),
        _native._ptr(W), _native._ptr(H), int(device)))
    return _unstack(ranks, W, H)


def consensus_sweep(V: np.ndarray, ranks: Iterable[int] = range(2, 11), n_runs: int = 64,
                    max_iter: int = 200, *, precision: str = "fp32", base_seed: int = 2024,
                    batched: bool = True, device: int = 0, metrics: bool = True) -> dict:
    """Consensus clustering for every rank in ``ranks`` (n_runs brunet
    restarts each, the reference's run_with_consensus per rank).

    Returns ``{"per_rank": {k: {"consensus", "cophenetic", "dispersion"}},
    "W", "H", "ranks", "solve_seconds", "consensus_seconds"}`` with the
    stacked factors of all solves (rank-major, run-minor).  The consensus
    matrices and, with ``metrics``, their cophenetic correlation and
    dispersion are computed on the GPU (``consensus_seconds``)."""
    import torch

    ranks = [int(k) for k in ranks]
    V = np.ascontiguousarray(np.asarray(V, dtype=np.float64))
    n, p = V.shape
    starts = []
    for k in ranks:
        starts.extend(restart_starts(V, k, n_runs, base_seed))
    rk, W0, H0 = _stack(starts)
    dev = torch.device("cuda", device)
    dV = torch.from_numpy(V).to(dev)
    dW = torch.from_numpy(W0).to(dev)
    dH = torch.from_numpy(H0).to(dev)
    ctx = _native.Context(device)
    lib = _native.load()
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    if batched:
        _native.check(lib.nmfcu_run_batch_device(
            ctx.handle, _native.parse_method("brunet"), _native.PRECISIONS[precision],
            int(max_iter), n, p, ctypes.c_void_p(dV.data_ptr()), p, len(rk), _ranks_ptr(rk),
            ctypes.c_void_p(dW.data_ptr()), ctypes.c_void_p(dH.data_ptr()),
            ctypes.c_void_p(stream.cuda_stream)))
    else:
        opts = _native.default_options()
        opts.method = _native.parse_method("brunet")
        opts.precision = _native.PRECISIONS[precision]
        opts.max_iter = int(max_iter)
        opts.refine_iters = 0
        opts.device = int(device)
        off = 0
        for r in rk:
            r = int(r)
            w = dW[:, off:off + r].contiguous()
            h = dH[off:off + r].contiguous()
            ctx.run(opts, n, p, r, dV.data_ptr(), _native.F64, p, w.data_ptr(), h.data_ptr(),
                    stream=stream.cuda_stream)
            dW[:, off:off + r] = w
            dH[off:off + r] = h
            off += r
    torch.cuda.synchronize(dev)
    out = {"per_rank": {}, "solve_seconds": time.perf_counter() - t0}
    cons = torch.empty((len(ranks), p, p), dtype=torch.float32, device=dev)
    t1 = time.perf_counter()
    mats, stats = {}, {}
    for ci, k in enumerate(ranks):
        sel = np.arange(ci * n_runs, (ci + 1) * n_runs, dtype=np.int32)
        _native.check(lib.nmfcu_consensus_device(
            ctx.handle, p, len(rk), _ranks_ptr(rk), ctypes.c_void_p(dH.data_ptr()), len(sel),
            _ranks_ptr(sel), ctypes.c_void_p(cons[ci].data_ptr()),
            ctypes.c_void_p(stream.cuda_stream)))
    if metrics:
        for k, st in zip(ranks, consensus_stats_batch(cons, ctx)):
            stats[k] = st
    for ci, k in enumerate(ranks):
        mats[k] = cons[ci].cpu().numpy()
    torch.cuda.synchronize(dev)
    out["consensus_seconds"] = time.perf_counter() - t1
    for k in ranks:
        entry = {"consensus": mats[k]}
        if metrics:
            entry["cophenetic"], entry["dispersion"] = stats[k]
        out["per_rank"][k] = entry
    out["W"] = dW.cpu().numpy()
    out["H"] = dH.cpu().numpy()
    out["ranks"] = rk
    ctx.close()
    return out
