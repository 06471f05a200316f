"""One NMF solve split by columns of V over several GPUs (one process a GPU).

The reference has a single-process loop (nmf_run_lee lib.rs:1589-1647,
nmf_run_brunet :1529-1586, nmf_run_hals :638-688, nmf_run_dnmf :827-906).
Its H update is local to each column of V given W; its W update needs, over
all columns, the W contraction (V H^T, or sum_j V_ij / (WH)_ij H_kj for
brunet), H H^T and rowSums(H).  So rank q holds V[:, c0:c1] (only its
columns, in its own HBM), its H columns and a copy of W; per iteration it
updates its H, computes its terms of those three sums into one flat device
buffer, the ranks sum the buffer with one all-reduce (NCCL over
NVLink/NVSwitch; about n r 8 bytes -- 3.2 MB at 20000 x 200000 rank 20), and
every rank applies the same W update to its copy.  The stationary stop's
objective is one more all-reduce of a scalar, so every rank takes the same
stop decision at the same iteration.

``run_shard`` drives any object with the step interface of ``DeviceShard``
(the CUDA library's half-steps, ``nmfcu_shard_*``) and a ``reduce`` callable
that sums tensors over the ranks in place.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Optional

import numpy as np

from . import _native

HALF_STEP, W_UPDATE, OBJECTIVE, STOP = 0, 1, 2, 3
ALIGN = 16  # column block boundaries in elements: 128-byte aligned shard bases


def split_columns(p: int, world: int, rank: int, align: int = ALIGN) -> tuple[int, int]:
    """Column range [c0, c1) of rank `rank` among `world`: contiguous blocks of
    near-equal width whose boundaries fall on multiples of `align` columns
    (so each shard's first element keeps V's alignment)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    units = -(-p // align)
    lo = units * rank // world
    hi = units * (rank + 1) // world
    return min(p, lo * align), min(p, hi * align)


def run_shard(shard, reduce: Callable, max_iter: int, stationary: bool) -> tuple[int, bool]:
    """Drive one rank's shard through the loop.  `reduce(t)` sums tensor t
    over the ranks in place.  Every rank takes the same collective steps in
    the same order (the stop decision follows an all-reduced scalar).
    Returns (iterations, stopped early)."""
    if stationary:
        shard.step(OBJECTIVE)
        reduce(shard.objective)
        shard.step(STOP)
        n_iter, stopped = shard.status()
        if stopped:
            return n_iter, True
    for _ in range(max_iter):
        shard.step(HALF_STEP)
        reduce(shard.reduce_buffer)
        shard.step(W_UPDATE)
        if stationary:
            shard.step(OBJECTIVE)
            reduce(shard.objective)
            shard.step(STOP)
            n_iter, stopped = shard.status()
            if stopped:
                return n_iter, True
    n_iter, _ = shard.status()
    return n_iter, False


class DeviceShard:
    """This rank's column shard on the CUDA library (``nmfcu_shard_*``).

    V_local: f64 torch tensor on the GPU, n x p_local, unit column stride,
    base and row pitch 16-byte aligned (a column block from ``split_columns``
    of a V with an even pitch qualifies).  W0 (n x r) and H0_local
    (r x p_local) are copied in."""

    def __init__(self, V_local, W0, H0_local, opts: "_native.Options", stream=None):
        import torch

        self.torch = torch
        self.lib = _native.load()
        if V_local.device.type != "cuda" or V_local.dtype != torch.float64:
            raise ValueError("V_local must be an f64 CUDA tensor")
        self.device = V_local.device
        n, p_local = V_local.shape
        r = W0.shape[1]
        self.n, self.p, self.r = n, p_local, r
        self.stream = stream or torch.cuda.current_stream(self.device)
        self.ctx = _native.Context(self.device.index or 0)
        f64 = dict(dtype=torch.float64, device=self.device)
        self.W0 = torch.as_tensor(np.ascontiguousarray(W0) if isinstance(W0, np.ndarray) else W0,
                                  **f64).contiguous()
        self.H0 = torch.as_tensor(np.ascontiguousarray(H0_local)
                                  if isinstance(H0_local, np.ndarray) else H0_local,
                                  **f64).contiguous()
        self.reduce_buffer = torch.zeros(int(self.lib.nmfcu_shard_reduce_len(n, r)), **f64)
        self.objective = torch.zeros(1, **f64)
        self.V = V_local
        self.opts = opts
        h = ctypes.c_void_p()
        _native.check(self.lib.nmfcu_shard_create(
            self.ctx.handle, ctypes.byref(opts), n, p_local, r,
            ctypes.c_void_p(V_local.data_ptr() if p_local else None),
            max(V_local.stride(0), p_local), ctypes.c_void_p(self.W0.data_ptr()),
            ctypes.c_void_p(self.H0.data_ptr() if p_local else None),
            ctypes.c_void_p(self.reduce_buffer.data_ptr()),
            ctypes.c_void_p(self.objective.data_ptr()), ctypes.byref(h),
            ctypes.c_void_p(self.stream.cuda_stream)))
        self.handle = h

    def step(self, phase: int):
        _native.check(self.lib.nmfcu_shard_step(self.handle, int(phase),
                                                ctypes.c_void_p(self.stream.cuda_stream)))

    def status(self) -> tuple[int, bool]:
        ni = ctypes.c_int64(0)
        stopped = ctypes.c_int32(0)
        _native.check(self.lib.nmfcu_shard_status(self.handle, ctypes.byref(ni),
                                                  ctypes.byref(stopped),
                                                  ctypes.c_void_p(self.stream.cuda_stream)))
        return int(ni.value), bool(stopped.value)

    def result(self):
        """(W, H_local, deviances) as torch tensors on the device."""
        torch = self.torch
        f64 = dict(dtype=torch.float64, device=self.device)
        W = torch.empty((self.n, self.r), **f64)
        H = torch.empty((self.r, self.p), **f64)
        dev = torch.empty(max(int(self.opts.max_iter) + 1, 1), **f64)
        nd, ni = ctypes.c_int64(0), ctypes.c_int64(0)
        _native.check(self.lib.nmfcu_shard_result(
            self.handle, ctypes.c_void_p(W.data_ptr()),
            ctypes.c_void_p(H.data_ptr() if self.p else None), ctypes.c_void_p(dev.data_ptr()),
            ctypes.byref(nd), ctypes.byref(ni), ctypes.c_void_p(self.stream.cuda_stream)))
        return W, H, dev[: nd.value]

    def close(self):
        if getattr(self, "handle", None):
            self.lib.nmfcu_shard_destroy(self.handle)
            self.handle = None
            self.ctx.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def torch_reduce(group=None) -> Callable:
    """Sum over the ranks of `group` with torch.distributed (NCCL for CUDA
    tensors); the identity when torch.distributed is not initialised."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return lambda t: None

    def reduce(t):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)

    return reduce


def nmf_sharded(V_local, rank: int, method: str = "lee", *, W0, H0_local, max_iter: int = 2000,
                eps: float = 1e-9, rescale: bool = True, sparsity: float = 0.01,
                stop: str = "max_iter", stationary_th: float = float(np.finfo(np.float64).eps),
                check_interval: int = 50, check_niter: int = 10, precision: str = "fp64",
                refine_iters: int = 2, group=None, reduce: Optional[Callable] = None):
    """One solve over the ranks of `group`: this rank passes its column block
    V_local (device tensor, see ``DeviceShard``), the full W0 (the same on
    every rank) and its columns of H0.  Returns (W, H_local, n_iter,
    deviances) as device tensors; W is the same on every rank."""
    o = _native.default_options()
    o.method = _native.parse_method(method)
    o.stop = _native.parse_stop(stop)
    o.precision = _native.PRECISIONS[str(precision).lower()]
    o.max_iter = int(max_iter)
    o.eps = float(eps)
    o.rescale = int(bool(rescale))
    if o.method == _native.DNMF:
        o.sparsity_h = o.sparsity_w = float(sparsity)
    o.stationary_th = float(stationary_th)
    o.check_interval = int(check_interval)
    o.check_niter = int(check_niter)
    o.refine_iters = int(refine_iters)
    o.device = V_local.device.index or 0
    sh = DeviceShard(V_local, W0, H0_local, o)
    try:
        run_shard(sh, reduce or torch_reduce(group), o.max_iter, o.stop == 1)
        W, H, dev = sh.result()
        n_iter, _ = sh.status()
    finally:
        sh.close()
    return W, H, n_iter, dev
