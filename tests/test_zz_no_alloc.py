"""The allocation-free objective entry point (nmfcu_objective_noalloc).

It exists for callers that may not allocate device memory while they run,
such as a server that reserves all of its GPU memory up front or code running
under another framework's memory pool. Its scratch is a fixed array inside
the library. These tests call it through the C ABI on device buffers and
compare it with the allocating entry points (nmfcu_divergence /
nmfcu_distance), two calls in a row, within the objective tolerance of the
other parity tests (1e-12 relative).

The file name makes pytest collect it last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import rel

import nmf_rs
from nmf_rs import _native, synthetic

pytestmark = pytest.mark.gpu

OBJ_TOL = 1e-12


def _noalloc(kind, V, W, H, pad=0, side_stream=False):
    """One call on device copies of V, W, H; returns the device result.

    pad > 0 embeds V in a wider device buffer (leading dimension p + pad);
    side_stream runs the call on a fresh stream instead of the current one."""
    import torch

    lib = _native.load()
    n, p = V.shape
    r = W.shape[1]
    ldv = p + pad
    Vbuf = np.full((n, ldv), np.nan)  # the padding must never be read
    Vbuf[:, :p] = V
    dV = torch.from_numpy(Vbuf).cuda()
    dW = torch.from_numpy(np.ascontiguousarray(W)).cuda()
    dH = torch.from_numpy(np.ascontiguousarray(H)).cuda()
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream() if side_stream else torch.cuda.current_stream()
    if side_stream:
        stream.wait_stream(torch.cuda.current_stream())
    _native.check(lib.nmfcu_objective_noalloc(
        kind, n, p, r, ctypes.c_void_p(dV.data_ptr()), ldv, ctypes.c_void_p(dW.data_ptr()),
        ctypes.c_void_p(dH.data_ptr()), ctypes.c_void_p(out.data_ptr()),
        ctypes.c_void_p(stream.cuda_stream)))
    stream.synchronize()
    return float(out.item())


def test_noalloc_matches_allocating_entry_points_twice():
    cases = [
        synthetic.counts_matrix(700, 900, 6, 0.3, seed=5),
        synthetic.counts_matrix(301, 77, 3, 0.3, seed=6),  # fewer rows: fewer partials
    ]
    for call, V in enumerate(cases):
        r = 7 if call == 0 else 19
        W, H = nmf_rs.random_init(V, r, seed=call)
        got_kl = _noalloc(_native.OBJECTIVE_KL, V, W, H)
        got_fro = _noalloc(_native.OBJECTIVE_FROBENIUS, V, W, H)
        assert rel(got_kl, _native.divergence(V, W, H)) <= OBJ_TOL
        assert rel(got_fro, _native.distance(V, W, H)) <= OBJ_TOL


def test_noalloc_rejects_rows_beyond_scratch():
    lib = _native.load()
    out = ctypes.c_double(0.0)
    with pytest.raises(ValueError, match="no-allocation scratch limit"):
        _native.check(lib.nmfcu_objective_noalloc(
            _native.OBJECTIVE_KL, _native.NOALLOC_MAX_ROWS + 1, 4, 2, None, 4, None, None,
            ctypes.addressof(out), None))


def test_noalloc_padded_rows_and_side_stream():
    """V inside a wider buffer (ldv > p; the padding holds NaN, so reading it
    would show), on a stream other than the current one."""
    V = synthetic.counts_matrix(333, 250, 4, 0.3, seed=8)
    W, H = nmf_rs.random_init(V, 9, seed=3)
    for kind, ref in ((_native.OBJECTIVE_KL, _native.divergence(V, W, H)),
                      (_native.OBJECTIVE_FROBENIUS, _native.distance(V, W, H))):
        assert rel(_noalloc(kind, V, W, H, pad=13), ref) <= OBJ_TOL
        assert rel(_noalloc(kind, V, W, H, pad=6, side_stream=True), ref) <= OBJ_TOL


def test_noalloc_empty_inputs_write_zero_without_reading_factors():
    """n == 0 or p == 0: the objective is 0 and the (NULL) V, W, H are not
    read.  The output starts as NaN, so a skipped write would show."""
    import torch

    lib = _native.load()
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    for n, p in ((0, 40), (25, 0), (0, 0)):
        for kind in (_native.OBJECTIVE_KL, _native.OBJECTIVE_FROBENIUS):
            out.fill_(float("nan"))
            _native.check(lib.nmfcu_objective_noalloc(
                kind, n, p, 3, None, max(p, 0), None, None, ctypes.c_void_p(out.data_ptr()),
                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
            torch.cuda.synchronize()
            assert float(out.item()) == 0.0
