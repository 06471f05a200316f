"""Seeded synthetic count matrices with single-cell-like structure.

The reference benchmarks on log-normalised single-cell data (pbmc8k,
2000 genes x 7750 cells).  This generator produces matrices of any shape
with the same kind of structure, from ``numpy.random.default_rng(seed)``:

  W_true (n x k) ~ Gamma(0.5, 1) with 70 % of its entries set to zero,
  H_true (k x p) with Dirichlet(alpha 1_k) columns,
  library sizes L_j ~ LogNormal(mu=7, sigma=0.5),
  counts ~ Poisson(W_true H_true diag(L)),
  every non-empty column scaled to sum 1e4, then V = log1p(counts).

Starting points are ``random_init(V, rank, seed)``: U(0, max V), W first.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def counts_matrix(n: int, p: int, k: int, alpha: float, seed: int, *, zero_frac: float = 0.7,
                  mu: float = 7.0, sigma: float = 0.5, target_sum: float = 1e4) -> np.ndarray:
    """V (n x p, f64, C-contiguous) from the generator described above."""
    gen = np.random.default_rng(seed)
    w_true = gen.gamma(0.5, 1.0, size=(n, k))
    w_true[gen.random((n, k)) < zero_frac] = 0.0
    h_true = gen.dirichlet(np.full(k, float(alpha)), size=p).T
    lib_size = gen.lognormal(mu, sigma, size=p)
    counts = gen.poisson((w_true @ h_true) * lib_size[None, :]).astype(np.float64)
    col = counts.sum(axis=0)
    scale = np.divide(target_sum, col, out=np.zeros_like(col), where=col > 0)
    return np.ascontiguousarray(np.log1p(counts * scale[None, :]))


def starting_point(V: np.ndarray, rank: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """(W0, H0) ~ U(0, max V) with W drawn before H (the reference's order)."""
    from . import random_init

    return random_init(V, rank, seed=seed)


@dataclass(frozen=True)
class Workload:
    """One benchmark configuration: shape, ground-truth rank, Dirichlet
    concentration, factorisation rank, iterations and method."""

    name: str
    n: int
    p: int
    k: int
    alpha: float
    rank: int
    iters: int
    method: str
    seed: int = 0


# The configurations the engine is measured on.
PBMC_SUBSET = Workload("lee-1500x3000-r8", 1500, 3000, 8, 0.3, 8, 100, "lee")
PBMC8K_SHAPE = Workload("brunet-2000x7750-r10", 2000, 7750, 10, 0.2, 10, 100, "brunet")
ATLAS = Workload("atlas-20000x200000-r20", 20000, 200000, 20, 0.2, 20, 25, "lee")
CONSENSUS = Workload("consensus-2000x5000-k2..10", 2000, 5000, 6, 0.2, 10, 200, "brunet")


def make(w: Workload) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(V, W0, H0) for a workload."""
    V = counts_matrix(w.n, w.p, w.k, w.alpha, w.seed)
    W0, H0 = starting_point(V, w.rank, w.seed)
    return V, W0, H0


def device_workload(n: int, p: int, k: int, alpha: float, rank: int, seed: int, device):
    """The same generator on the device (torch's RNG, so not the same draws
    as :func:`counts_matrix`), for shapes too large to build on the host in
    reasonable time.  Returns (V64, ld64, V32, ld32, W0, H0): V in f64 with
    its leading dimension padded to 16 elements and in f32 padded to 32
    (zeros in the padding), and a U(0, max V) start."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    f64 = torch.float64
    w_true = torch._standard_gamma(torch.full((n, k), 0.5, dtype=f64, device=device),
                                   generator=g)
    w_true[torch.rand((n, k), generator=g, device=device, dtype=f64) < 0.7] = 0.0
    ld64 = (p + 15) // 16 * 16
    ld32 = (p + 31) // 32 * 32
    V64 = torch.zeros((n, ld64), dtype=f64, device=device)
    chunk = 8192
    for c0 in range(0, p, chunk):
        c = min(chunk, p - c0)
        h = torch._standard_gamma(torch.full((k, c), float(alpha), dtype=f64, device=device),
                                  generator=g)
        h = h / h.sum(0, keepdim=True).clamp_min(1e-300)
        lib = torch.empty(c, dtype=f64, device=device).log_normal_(7.0, 0.5, generator=g)
        lam = (w_true @ h) * lib[None, :]
        counts = torch.poisson(lam, generator=g)
        col = counts.sum(0, keepdim=True)
        scale = torch.where(col > 0, 1e4 / col.clamp_min(1e-300), torch.zeros_like(col))
        V64[:, c0:c0 + c] = torch.log1p(counts * scale)
        del h, lam, counts
    V32 = torch.zeros((n, ld32), dtype=torch.float32, device=device)
    V32[:, :p] = V64[:, :p].float()
    vmax = float(V64[:, :p].max())
    W0 = torch.rand((n, rank), generator=g, device=device, dtype=f64) * vmax
    H0 = torch.rand((rank, p), generator=g, device=device, dtype=f64) * vmax
    return V64, ld64, V32, ld32, W0, H0
