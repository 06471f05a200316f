"""nmf_rs -- non-negative matrix factorisation on one NVIDIA B200.

Drop-in for the Python surface of omicverse/rust-NMF
(``python/nmf_rs/__init__.py``): the same ``nmf()``, ``NMFResult``,
single-step updates, ``random_init``, ``nndsvd_init``, ``smoothing_matrix``
and ``set_num_threads``, with the iteration loop running as hand-written
sm_100a CUDA kernels behind the C ABI of ``include/nmfcu.h``.

Built methods: ``brunet`` (KL), ``lee`` (Frobenius), ``offset``, ``nsNMF``,
``hals``, ``ehals``, ``dnmf``, ``lsnmf`` (weighted) and the Kim-Park
``snmf/r`` / ``snmf/l`` (FCNNLS), each with ``stop='max_iter'`` or
``'stationary'`` (snmf runs max_iter iterations, as the reference does);
lsnmf and snmf in FP64 only.  There is no CPU fallback: without the CUDA library
or a GPU every compute call raises ``RuntimeError``.

Engine extensions (keyword-only, defaults keep the reference's behaviour):
``precision='fp64'|'fp32'`` and ``refine_iters`` on :func:`nmf`.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _native

__all__ = [
    "NMFResult",
    "nmf",
    "update_h_brunet",
    "update_w_brunet",
    "update_h_lee",
    "update_w_lee",
    "smoothing_matrix",
    "random_init",
    "nndsvd_init",
    "cv_rank",
    "set_num_threads",
]


# =============================================================================
# Result type (python/nmf_rs/__init__.py:59-99)
# =============================================================================

@dataclass
class NMFResult:
    """Outcome of an NMF run: ``W`` (n x rank), ``H`` (rank x p), ``n_iter``,
    ``deviances`` (objective per iteration; empty for ``stop='max_iter'``),
    ``method`` and ``offset`` (only for the offset algorithm)."""

    W: np.ndarray
    H: np.ndarray
    n_iter: int
    deviances: np.ndarray = field(default_factory=lambda: np.empty(0, dtype=np.float64))
    method: str = "brunet"
    offset: Optional[np.ndarray] = None

    @property
    def basis(self) -> np.ndarray:
        return self.W

    @property
    def coef(self) -> np.ndarray:
        return self.H

    def fitted(self) -> np.ndarray:
        """The model estimate W H (plus the offset column, when present)."""
        wh = self.W @ self.H
        if self.offset is not None:
            wh = wh + self.offset[:, None]
        return wh

    def __repr__(self) -> str:
        return (
            f"NMFResult(method='{self.method}', n={self.W.shape[0]}, "
            f"p={self.H.shape[1]}, rank={self.W.shape[1]}, n_iter={self.n_iter})"
        )


# =============================================================================
# Initialisation (python/nmf_rs/__init__.py:110-219)
# =============================================================================

def random_init(V: np.ndarray, rank: int, seed: Optional[int] = None, *,
                max_value: Optional[float] = None) -> tuple[np.ndarray, np.ndarray]:
    """(W0, H0) drawn U(0, max V) from ``numpy.random.default_rng(seed)``:
    W (n x rank) first, then H (rank x p) -- the reference's stream order,
    so the same seed gives the same starting point."""
    n, p = V.shape
    gen = np.random.default_rng(seed)
    if max_value is not None:
        top = float(max_value)
    else:
        top = float(np.max(V)) if V.size else 1.0
    W0 = gen.uniform(0.0, top, size=(n, rank))
    H0 = gen.uniform(0.0, top, size=(rank, p))
    return W0, H0


def nndsvd_init(V: np.ndarray, rank: int, *, fill: str = "mean", seed: int = 0,
                n_oversamples: int = 10, device: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """NNDSVD start (Boutsidis & Gallopoulos 2008, "SVD based initialization:
    A head start for nonnegative matrix factorization"), the reference's
    ``nndsvd_init`` (python/nmf_rs/__init__.py:129-219).

    A rank-``rank`` randomized SVD of V -- the algorithm of scikit-learn's
    ``randomized_svd`` with ``random_state=seed``, its passes over V on the
    GPU (``nmf_rs.nndsvd``) -- is turned into non-negative factors: the
    leading pair by absolute value, every later pair by keeping whichever
    sign-split half (u+, v+) or (u-, v-) has the larger norm product, scaled
    to carry sqrt(sigma * that product).  Zeros are then kept (``'zero'``),
    raised to 1e-9 (``'eps'``) or replaced by mean(V) (``'mean'``, NNDSVDa).
    ``device`` (engine extension) selects the GPU.
    """
    V = np.asarray(V, dtype=np.float64)
    if (V < 0).any():
        raise ValueError("V must be non-negative for NNDSVD initialisation.")
    if fill not in ("zero", "mean", "eps"):
        raise ValueError(f"unknown fill mode '{fill}': supported zero / mean / eps")
    if _native.device_count() < 1:
        raise RuntimeError("nndsvd_init() runs its passes over V on a CUDA device; none is visible")
    from . import nndsvd

    Vd = nndsvd.upload(V, int(device))
    W, H = nndsvd.nndsvd_device(Vd, int(rank), fill=fill, seed=int(seed),
                                n_oversamples=int(n_oversamples))
    return W.cpu().numpy(), H.cpu().numpy()


# =============================================================================
# Single-step updates (python/nmf_rs/__init__.py:243-264)
# =============================================================================

def _f64_c(arr, name: str) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(arr, dtype=np.float64))
    if a.ndim != 2:
        raise ValueError(f"{name} must be 2-D, got shape {a.shape}")
    return a


def update_h_brunet(V: np.ndarray, W: np.ndarray, H: np.ndarray) -> np.ndarray:
    """One brunet (KL) update of H (R ``std.divergence.update.h``)."""
    return _native.py_divergence_update_h(_f64_c(V, "V"), _f64_c(W, "W"), _f64_c(H, "H"))


def update_w_brunet(V: np.ndarray, W: np.ndarray, H: np.ndarray) -> np.ndarray:
    """One brunet (KL) update of W (R ``std.divergence.update.w``)."""
    return _native.py_divergence_update_w(_f64_c(V, "V"), _f64_c(W, "W"), _f64_c(H, "H"))


def update_h_lee(V: np.ndarray, W: np.ndarray, H: np.ndarray, eps: float = 1e-9) -> np.ndarray:
    """One lee (Frobenius) update of H (R ``std.euclidean.update.h``)."""
    return _native.py_euclidean_update_h(_f64_c(V, "V"), _f64_c(W, "W"), _f64_c(H, "H"),
                                         float(eps))


def update_w_lee(V: np.ndarray, W: np.ndarray, H: np.ndarray, eps: float = 1e-9) -> np.ndarray:
    """One lee (Frobenius) update of W (R ``std.euclidean.update.w``)."""
    return _native.py_euclidean_update_w(_f64_c(V, "V"), _f64_c(W, "W"), _f64_c(H, "H"),
                                         float(eps))


def smoothing_matrix(rank: int, theta: float) -> np.ndarray:
    """nsNMF smoothing matrix S = (1 - theta) I + (theta / r) 1 1^T."""
    return _native.py_smoothing_matrix(int(rank), float(theta))


def set_num_threads(n: int) -> bool:
    """Accepted for compatibility; the GPU engine has no CPU pool (False)."""
    return _native.set_num_threads(int(n))


def cv_rank(V: np.ndarray, ranks: Sequence[int], *, method: str = "hals", n_folds: int = 4,
            mask_frac: float = 0.05, max_iter: int = 100, init: str = "nndsvd", seed: int = 0,
            num_threads: Optional[int] = None, device: int = 0, **nmf_kwargs):
    """Cross-validated rank selection by held-out reconstruction error, the
    reference's ``cv_rank`` (python/nmf_rs/__init__.py:273-355).

    For every rank and fold a fresh seed from ``default_rng(seed)`` draws a
    mask holding out ``mask_frac`` of V's entries; the fold is fitted with
    the weighted ``lsnmf`` method (held-out entries weigh 0) from an NNDSVD
    (``init='nndsvd'``) or uniform start of the masked V, and scored by the
    0.5 weighted squared residual on the kept entries and the mean squared
    error on the held-out ones.  ``method`` is accepted as in the reference
    (which does not use it).  Returns a pandas DataFrame with columns rank,
    fold, train_loss, test_mse.
    """
    import pandas as pd

    V = _f64_c(V, "V")
    if (V < 0).any():
        raise ValueError("V must be non-negative")
    n, p = V.shape
    master = np.random.default_rng(seed)
    rows = []
    for k in ranks:
        for fold in range(n_folds):
            fold_seed = int(master.integers(0, 2**31 - 1))
            keep = np.random.default_rng(fold_seed).random((n, p)) > mask_frac
            weight = keep.astype(np.float64)
            V_train = V * weight
            if init == "nndsvd":
                W0, H0 = nndsvd_init(V_train, k, fill="mean", seed=fold_seed, device=device)
            else:
                W0, H0 = random_init(V_train, k, seed=fold_seed)
            res = nmf(V_train, rank=k, method="ls-nmf", W0=W0, H0=H0, weight=weight,
                      max_iter=max_iter, num_threads=num_threads, device=device, **nmf_kwargs)
            recon = res.fitted()
            train_loss = 0.5 * float((((V - recon) * weight) ** 2).sum())
            held = ~keep
            test_mse = float(((V[held] - recon[held]) ** 2).mean())
            rows.append({"rank": int(k), "fold": fold, "train_loss": train_loss,
                         "test_mse": test_mse})
    return pd.DataFrame(rows)


# =============================================================================
# Top-level driver (python/nmf_rs/__init__.py:362-568)
# =============================================================================

_METHOD_ALIASES = {
    "brunet": "brunet", "kl": "brunet",
    "lee": "lee", "frobenius": "lee", "euclidean": "lee",
    "offset": "offset",
    "nsnmf": "nsnmf", "ns": "nsnmf", "ns_nmf": "nsnmf",
    "hals": "hals",
    "ehals": "ehals", "e-hals": "ehals", "extrap_hals": "ehals",
    "dnmf": "dnmf", "diag_nmf": "dnmf", "rcppml": "dnmf",
    "ls-nmf": "lsnmf", "lsnmf": "lsnmf",
    "snmf/r": "snmf/r", "snmf_r": "snmf/r", "snmfr": "snmf/r",
    "snmf/l": "snmf/l", "snmf_l": "snmf/l", "snmfl": "snmf/l",
}


def _regularisation(method: str, sparsity: float, smoothness: float):
    """Per-method routing of ``sparsity``/``smoothness`` to the L1/L2 terms
    of each factor (python/nmf_rs/__init__.py:528-538)."""
    if method == "snmf/r":
        return float(sparsity), 0.0, 0.0, float(smoothness)
    if method == "snmf/l":
        return 0.0, float(sparsity), float(smoothness), 0.0
    if method == "dnmf":
        return float(sparsity), float(sparsity), 0.0, 0.0
    return 0.0, 0.0, 0.0, 0.0


# Methods that run on a sparse V (nmfcu_run_csr).
_SPARSE_METHODS = {"lee", "brunet", "hals", "dnmf"}


def _is_sparse(V) -> bool:
    try:
        import scipy.sparse as sp
    except ImportError:  # pragma: no cover - scipy ships with the engine's deps
        return False
    return sp.issparse(V)


def _prepare(V, rank, method, W0, H0, seed, offset, weight, sparsity, smoothness):
    """nmf()'s argument handling before the native call, in the reference's
    order (python/nmf_rs/__init__.py:487-538): method aliases, V >= 0, a
    random start for a missing W0/H0, shape checks, sparsity routing."""
    method_norm = _METHOD_ALIASES.get(method.lower())
    if method_norm is None:
        raise ValueError(
            f"unknown method '{method}'. supported: brunet, lee, offset, nsNMF "
            "(plus aliases KL/Frobenius/ns).")
    if _is_sparse(V):
        # Engine extension: a scipy.sparse V stays sparse (the stored entries
        # are all the loop reads); the reference densifies it here.
        if method_norm not in _SPARSE_METHODS:
            raise NotImplementedError(
                f"method '{method}' needs a dense V; a sparse V runs "
                + ", ".join(sorted(_SPARSE_METHODS)))
        V_arr = V.tocsr().astype(np.float64)
        if V_arr.ndim != 2:
            raise ValueError(f"V must be 2-D, got shape {V_arr.shape}")
        if (V_arr.data < 0).any():
            raise ValueError("V must be non-negative.")
        vmax = float(V_arr.max()) if V_arr.shape[0] * V_arr.shape[1] else 1.0
    else:
        V_arr = _f64_c(V, "V")
        if (V_arr < 0).any():
            raise ValueError("V must be non-negative.")
        vmax = None
    n, p = V_arr.shape
    if W0 is None or H0 is None:
        W0_, H0_ = random_init(V_arr, rank, seed=seed, max_value=vmax)
        W0 = W0_ if W0 is None else W0
        H0 = H0_ if H0 is None else H0
    W0 = _f64_c(W0, "W0")
    H0 = _f64_c(H0, "H0")
    if W0.shape != (n, rank):
        raise ValueError(f"W0.shape {W0.shape} != ({n}, {rank})")
    if H0.shape != (rank, p):
        raise ValueError(f"H0.shape {H0.shape} != ({rank}, {p})")
    offset_arr = None
    if offset is not None:
        offset_arr = np.ascontiguousarray(np.asarray(offset, dtype=np.float64))
        if offset_arr.shape != (n,):
            raise ValueError(f"offset.shape {offset_arr.shape} != ({n},)")
    weight_arr = None
    if weight is not None:
        weight_arr = np.ascontiguousarray(np.asarray(weight, dtype=np.float64))
        if weight_arr.shape != V_arr.shape:
            raise ValueError(f"weight.shape {weight_arr.shape} != V.shape {V_arr.shape}")
    sh, sw, gh, gw = _regularisation(method_norm, sparsity, smoothness)
    return method_norm, V_arr, W0, H0, offset_arr, weight_arr, (sh, sw, gh, gw)


def nmf(V: np.ndarray, rank: int, method: str = "brunet", *, W0: Optional[np.ndarray] = None,
        H0: Optional[np.ndarray] = None, seed: Optional[int] = None, max_iter: int = 2000,
        eps: float = 1e-9, rescale: bool = True, theta: float = 0.5,
        offset: Optional[np.ndarray] = None, weight: Optional[np.ndarray] = None,
        sparsity: float = 0.01, smoothness: float = 1.0, stop: str = "max_iter",
        stationary_th: float = float(np.finfo(np.float64).eps), check_interval: int = 50,
        check_niter: int = 10, num_threads: Optional[int] = None, precision: str = "fp64",
        refine_iters: int = 2, device: int = 0) -> NMFResult:
    """Factorise V ~ W H on the GPU.

    Arguments, defaults, validation order and result follow the reference's
    ``nmf()`` (python/nmf_rs/__init__.py:396-568): method aliases, a
    non-negativity check on V, ``random_init(V, rank, seed)`` for a missing
    W0/H0, shape checks, per-method sparsity routing.  ``num_threads`` is
    accepted and ignored.

    Engine extensions: ``precision='fp32'`` stores V in f32 for the two V
    contractions (f32 products, f64 reductions, f64 updates/objective/stop)
    and runs the last ``refine_iters`` iterations in full f64; ``device``
    selects the GPU.  A ``scipy.sparse`` V (any format; CSR is used) is
    factorised without densifying it, for lee, brunet, hals and dnmf in FP64:
    the passes read only its stored entries.
    """
    method_norm, V_arr, W0, H0, offset_arr, weight_arr, (sh, sw, gh, gw) = _prepare(
        V, rank, method, W0, H0, seed, offset, weight, sparsity, smoothness)
    run = _native.py_nmf_run_csr if _is_sparse(V_arr) else _native.py_nmf_run
    out = run(
        method_norm, V_arr, W0, H0, int(max_iter), eps=float(eps), rescale=bool(rescale),
        theta=float(theta), offset=offset_arr, weight=weight_arr, sparsity_h=sh,
        sparsity_w=sw, smoothness_h=gh, smoothness_w=gw, stop=stop,
        stationary_th=float(stationary_th), check_interval=int(check_interval),
        check_niter=int(check_niter),
        num_threads=int(num_threads) if num_threads is not None else None,
        precision=precision, refine_iters=int(refine_iters), device=int(device))
    return NMFResult(
        W=np.asarray(out["W"]),
        H=np.asarray(out["H"]),
        n_iter=int(out["n_iter"]),
        deviances=np.asarray(out["deviances"], dtype=np.float64),
        method=method_norm,
        offset=np.asarray(out["offset"]) if "offset" in out else None,
    )


from . import consensus, serve, synthetic  # noqa: E402,F401
