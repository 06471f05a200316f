"""NNDSVD start on the GPU.

``nndsvd_init`` of the reference (python/nmf_rs/__init__.py:129-219) takes a
rank-k randomized SVD of V with scikit-learn's ``randomized_svd``
(:172-174) and turns each singular pair into non-negative factors.  Here the
randomized SVD's passes over V -- the only work that grows with n x p -- run
as FP64 streaming passes of the CUDA library (``nmfcu_v_product_device``),
and the tall-skinny factorizations between them (LU with partial pivoting,
economic QR, the SVD of the small projected matrix) run on the same device
through torch.linalg (cuSOLVER).  V is read, never copied or transposed.

The randomized SVD follows Halko, Martinsson & Tropp, "Finding structure with
randomness" (2011), Algorithms 4.3/4.4, with the choices randomized_svd makes
(scikit-learn 1.9): l = k + n_oversamples Gaussian test vectors drawn by
``numpy.random.RandomState(seed).normal``; 7 power iterations when
k < 0.1 min(n, p), else 4, each product normalised by an LU factorization
(rows permuted back, "P L"); a final economic QR; the SVD of B = Q^T A;
A = V^T when n < p; signs fixed so that the largest-magnitude entry of each
singular vector (of U, or of V^T when A = V^T) is positive.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from . import _native


def _torch():
    import torch

    return torch


def _lu_pl(X):
    """P L of X = P L U (partial pivoting): the factor whose columns span X's
    range, rows returned to X's order."""
    torch = _torch()
    m, c = X.shape
    kk = min(m, c)
    LU, piv, _ = torch.linalg.lu_factor_ex(X)  # a singular U is fine here
    L = torch.tril(LU[:, :kk], diagonal=-1)
    L.diagonal().fill_(1.0)
    # LAPACK pivots: row i was swapped with row piv[i] - 1, i = 0, 1, ...
    perm = np.arange(m)
    for i, q in enumerate(piv.cpu().numpy().tolist()):
        q -= 1
        if q != i:
            perm[i], perm[q] = perm[q], perm[i]
    out = torch.empty_like(L)
    out[torch.from_numpy(perm).to(L.device)] = L
    return out


def _flip(U, Vt, u_based: bool):
    """Signs so that the largest-magnitude entry (the first one, on ties) of
    each left (u_based) or right singular vector is positive."""
    torch = _torch()
    if u_based:
        idx = torch.argmax(U.abs(), dim=0)
        signs = torch.sign(U[idx, torch.arange(U.shape[1], device=U.device)])
    else:
        idx = torch.argmax(Vt.abs(), dim=1)
        signs = torch.sign(Vt[torch.arange(Vt.shape[0], device=Vt.device), idx])
    return U * signs[None, :], Vt * signs[:, None]


def randomized_svd(V, k: int, *, n_oversamples: int = 10, seed: int = 0,
                   product: Optional[Callable] = None):
    """Rank-k randomized SVD of V (an f64 torch tensor, n x p, rows may be
    padded).  ``product(trans, X)`` returns V X (trans 0) or V^T X (trans 1);
    by default the CUDA library's streaming pass.  Returns (U, S, Vt) as torch
    tensors on V's device."""
    torch = _torch()
    n, p = V.shape
    if product is None:
        product = _device_product(V)
    l = k + n_oversamples
    n_iter = 7 if k < 0.1 * min(n, p) else 4
    transpose = n < p
    # A = V^T (p x n) when n < p, else V; A @ X and A^T @ X in V's terms.
    a_mul = (lambda X: product(1, X)) if transpose else (lambda X: product(0, X))
    at_mul = (lambda X: product(0, X)) if transpose else (lambda X: product(1, X))
    cols = n if transpose else p
    omega = np.random.RandomState(seed).normal(size=(cols, l))
    Q = torch.from_numpy(omega).to(device=V.device, dtype=torch.float64)
    normalise = _lu_pl if n_iter > 2 else (lambda X: X)
    for _ in range(n_iter):
        Q = normalise(a_mul(Q))
        Q = normalise(at_mul(Q))
    Q, _ = torch.linalg.qr(a_mul(Q), mode="reduced")
    B = at_mul(Q).T  # Q^T A
    Uhat, S, Vt = torch.linalg.svd(B, full_matrices=False)
    U = Q @ Uhat
    U, Vt = _flip(U, Vt, u_based=not transpose)
    if transpose:
        return Vt[:k].T, S[:k], U[:, :k].T
    return U[:, :k], S[:k], Vt[:k]


def _device_product(V):
    torch = _torch()
    if V.device.type != "cuda":
        raise RuntimeError("the NNDSVD passes over V run on a CUDA device")
    if V.dtype != torch.float64 or V.stride(1) != 1:
        raise ValueError("V must be an f64 tensor with unit column stride")
    ctx = _context(V.device.index or 0)
    n, p = V.shape

    def product(trans: int, X):
        X = X.contiguous()
        l = X.shape[1]
        out = torch.empty((p if trans else n, l), dtype=torch.float64, device=V.device)
        ctx.v_product(trans, n, p, l, V.data_ptr(), V.stride(0), X.data_ptr(), l,
                      out.data_ptr(), l, torch.cuda.current_stream(V.device).cuda_stream)
        return out

    return product


_CONTEXTS: dict = {}


def _context(device: int) -> "_native.Context":
    ctx = _CONTEXTS.get(device)
    if ctx is None:
        ctx = _CONTEXTS[device] = _native.Context(device)
    return ctx


def nndsvd_factors(V, U, S, Vt, fill: str):
    """Boutsidis & Gallopoulos (2008): the leading pair by absolute value,
    every later pair by the sign-split half (u+, v+) or (u-, v-) with the
    larger norm product (the positive half on ties), scaled to carry
    sqrt(sigma * that product); then the zero fill (``'zero'``: keep,
    ``'eps'``: raise to 1e-9, ``'mean'``: mean(V), NNDSVDa)."""
    torch = _torch()
    up, un = U.clamp(min=0.0), (-U).clamp(min=0.0)
    vp, vn = Vt.clamp(min=0.0), (-Vt).clamp(min=0.0)
    nup, nun = torch.linalg.vector_norm(up, dim=0), torch.linalg.vector_norm(un, dim=0)
    nvp, nvn = torch.linalg.vector_norm(vp, dim=1), torch.linalg.vector_norm(vn, dim=1)
    npos, nneg = nup * nvp, nun * nvn
    pos = npos >= nneg
    prod = torch.where(pos, npos, nneg)
    live = prod > 0
    sigma = torch.sqrt(S * prod)
    one = torch.ones_like(prod)
    wsc = torch.where(live, sigma / torch.where(pos, nup, nun).where(live, one), 0.0 * one)
    hsc = torch.where(live, sigma / torch.where(pos, nvp, nvn).where(live, one), 0.0 * one)
    W = torch.where(pos[None, :], up, un) * wsc[None, :]
    H = torch.where(pos[:, None], vp, vn) * hsc[:, None]
    root = torch.sqrt(S[0])
    W[:, 0] = root * U[:, 0].abs()
    H[0, :] = root * Vt[0, :].abs()
    if fill == "eps":
        W = W.clamp(min=1e-9)
        H = H.clamp(min=1e-9)
    elif fill == "mean":
        m = V.mean() if V.numel() else torch.zeros((), dtype=V.dtype, device=V.device)
        W = torch.where(W <= 0.0, m, W)
        H = torch.where(H <= 0.0, m, H)
    return W, H


class _Cusolver:
    """torch.linalg on CUDA through cuSOLVER for the scope (its default
    backend choice may pick MAGMA's batched routines for these tall, narrow
    factorizations); the caller's choice is restored on exit."""

    def __enter__(self):
        torch = _torch()
        self.prev = torch.backends.cuda.preferred_linalg_library()
        torch.backends.cuda.preferred_linalg_library("cusolver")

    def __exit__(self, *exc):
        _torch().backends.cuda.preferred_linalg_library(self.prev)
        return False


def nndsvd_device(V, rank: int, *, fill: str = "mean", seed: int = 0,
                  n_oversamples: int = 10, product: Optional[Callable] = None):
    """NNDSVD of a device-resident V (f64 torch tensor, n x p).  Returns
    (W0, H0) as torch tensors on V's device."""
    if fill not in ("zero", "mean", "eps"):
        raise ValueError(f"unknown fill mode '{fill}': supported zero / mean / eps")
    with _Cusolver():
        U, S, Vt = randomized_svd(V, int(rank), n_oversamples=int(n_oversamples),
                                  seed=int(seed), product=product)
        return nndsvd_factors(V, U, S, Vt, fill)


def upload(V: np.ndarray, device: int = 0):
    """V (host, f64) into device memory with a row pitch of a multiple of 16
    elements (128 bytes), as the streaming passes read it; returns the n x p
    view."""
    torch = _torch()
    n, p = V.shape
    ld = max(16, -(-p // 16) * 16)
    buf = torch.empty((n, ld), dtype=torch.float64, device=f"cuda:{device}")
    view = buf[:, :p]
    view.copy_(torch.from_numpy(np.ascontiguousarray(V, dtype=np.float64)))
    return view
