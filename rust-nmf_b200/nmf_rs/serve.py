"""Serving: many independent factorisations, submitted from any thread and
run concurrently on one GPU (``nmfcu_server_*``).

The reference has no server -- each ``nmf()`` call runs to completion on its
caller's thread (python/nmf_rs/__init__.py:396-568).  ``Server.submit`` takes
exactly ``nmf()``'s arguments, applies the same checks and routing, and
returns a ``Request`` whose ``result()`` is the ``NMFResult`` that ``nmf()``
would return for the same arguments.  The native server admits queued
requests as worker slots and device memory free up (the memory a request's
slot must add has to fit in the budget next to what every slot holds), so
requests that arrive while others run start as soon as there is room, and
their work overlaps on the device.

    with Server(slots=4) as srv:
        reqs = [srv.submit(V, 10, "brunet", W0=W0, H0=H0, max_iter=200) for V in mats]
        results = [r.result() for r in reqs]
        srv.stats()   # p50/p99 latency, iterations, memory
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _native

__all__ = ["Server", "Request"]

_QUEUED, _RUNNING, _DONE = 0, 1, 2


class Request:
    """One submitted factorisation.  Holds its host buffers until the result
    has been collected."""

    def __init__(self, server: "Server", rid: int, method: str, bufs: dict):
        self._server = server
        self.id = rid
        self._method = method
        self._bufs = bufs
        self._result = None
        self._error: Optional[BaseException] = None

    def state(self) -> str:
        if self._result is not None or self._error is not None:
            return "done"
        st = ctypes.c_int32(0)
        _native.check(self._server._lib.nmfcu_server_poll(self._server._h, self.id,
                                                          ctypes.byref(st)))
        return {_QUEUED: "queued", _RUNNING: "running", _DONE: "done"}[st.value]

    def done(self) -> bool:
        return self.state() == "done"

    def cancel(self) -> bool:
        """Cancel the request if it has not started; True if it was."""
        if self._result is not None or self._error is not None:
            return False
        st = self._server._lib.nmfcu_server_cancel(self._server._h, self.id)
        return st == _native.OK

    def result(self, timeout: Optional[float] = None):
        """Wait for the request (``timeout`` seconds, None: no limit) and return
        its ``NMFResult``; raises the request's error, ``TimeoutError`` if it
        has not finished in time."""
        from . import NMFResult

        if self._result is not None:
            return self._result
        if self._error is not None:
            raise self._error
        ni, nd = ctypes.c_int64(0), ctypes.c_int64(0)
        ms = -1 if timeout is None else max(0, int(timeout * 1000))
        st = self._server._lib.nmfcu_server_wait(self._server._h, self.id, ms, ctypes.byref(ni),
                                                 ctypes.byref(nd))
        if st == _native.TIMEOUT:
            raise TimeoutError(f"request {self.id} not finished within {timeout} s")
        try:
            _native.check(st)
        except BaseException as e:  # the id is released: keep the error
            self._error = e
            self._bufs = None
            raise
        b = self._bufs
        self._result = NMFResult(W=b["W"], H=b["H"], n_iter=int(ni.value),
                                 deviances=np.array(b["dev"][: nd.value], dtype=np.float64),
                                 method=self._method, offset=b.get("off"))
        self._bufs = None
        return self._result


class Server:
    """A request server on one GPU with continuous admission (requests run
    concurrently, each alone on its slot's stream).

    slots         concurrent requests (one engine context and stream each)
    budget_bytes  device memory the slots may hold (0: 90% of free memory)
    """

    def __init__(self, device: int = 0, slots: int = 4, budget_bytes: int = 0):
        self._lib = _native.load()
        h = ctypes.c_void_p()
        _native.check(self._lib.nmfcu_server_create(int(device), int(slots), int(budget_bytes),
                                                    ctypes.byref(h)))
        self._h = h
        self.device = int(device)

    def submit(self, V, rank: int, method: str = "brunet", *, W0=None, H0=None,
               seed: Optional[int] = None, max_iter: int = 2000, eps: float = 1e-9,
               rescale: bool = True, theta: float = 0.5, offset=None, weight=None,
               sparsity: float = 0.01, smoothness: float = 1.0, stop: str = "max_iter",
               stationary_th: float = float(np.finfo(np.float64).eps),
               check_interval: int = 50, check_niter: int = 10,
               num_threads: Optional[int] = None, precision: str = "fp64",
               refine_iters: int = 2) -> Request:
        """Queue ``nmf(V, rank, method, ...)``; arguments and checks as nmf()."""
        from . import _prepare

        method_norm, V_arr, W0, H0, offset_arr, weight_arr, (sh, sw, gh, gw) = _prepare(
            V, rank, method, W0, H0, seed, offset, weight, sparsity, smoothness)
        o, v, w0, h0, n, p, r = _native.build_run_options(
            method_norm, V_arr, W0, H0, int(max_iter), eps=float(eps), rescale=bool(rescale),
            theta=float(theta), offset=offset_arr, weight=weight_arr, sparsity_h=sh,
            sparsity_w=sw, smoothness_h=gh, smoothness_w=gw, stop=stop,
            stationary_th=float(stationary_th), check_interval=int(check_interval),
            check_niter=int(check_niter), num_threads=num_threads, precision=precision,
            refine_iters=int(refine_iters), device=self.device)
        W = np.empty((n, r), dtype=np.float64)
        H = np.empty((r, p), dtype=np.float64)
        cap = o.max_iter + 1
        dev = np.empty(cap, dtype=np.float64)
        rid = ctypes.c_int64(0)
        dp = _native._ptr
        bufs = {"V": v, "W0": w0, "H0": h0, "W": W, "H": H, "dev": dev, "opts": o}
        if method_norm == "offset":
            # The offset method also returns its row offsets (lib.rs:2161-2165).
            off = np.empty(n, dtype=np.float64)
            bufs.update(off=off, off0=offset_arr)
            _native.check(self._lib.nmfcu_server_submit_offset(
                self._h, ctypes.byref(o), n, p, r, dp(v), p, dp(w0), dp(h0),
                dp(offset_arr) if offset_arr is not None else None, dp(W), dp(H), dp(off),
                dp(dev), cap, ctypes.byref(rid)))
        else:
            _native.check(self._lib.nmfcu_server_submit(
                self._h, ctypes.byref(o), n, p, r, dp(v), p, dp(w0), dp(h0), dp(W), dp(H),
                dp(dev), cap, ctypes.byref(rid)))
        return Request(self, int(rid.value), method_norm, bufs)

    def stats(self) -> dict:
        st = _native.ServerStats()
        _native.check(self._lib.nmfcu_server_get_stats(self._h, ctypes.byref(st)))
        d = {name: getattr(st, name) for name, _ in _native.ServerStats._fields_}
        d["iters_per_s"] = (st.iterations / (st.wall_ms / 1000.0)) if st.wall_ms > 0 else 0.0
        return d

    def reset_stats(self) -> None:
        _native.check(self._lib.nmfcu_server_reset_stats(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.nmfcu_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
