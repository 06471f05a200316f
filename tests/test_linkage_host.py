"""The device consensus statistics' algorithm, restated in Python on CPU
(test infrastructure): the nearest-neighbour chain with the kernel's tie
rule and f64 Lance-Williams average update, and the cophenetic correlation
from the merges alone, against scipy's linkage + cophenet on consensus
matrices full of tied distances.  The GPU tests compare the kernel itself.
"""
from __future__ import annotations

import numpy as np
import pytest
from scipy.cluster.hierarchy import cophenet, linkage
from scipy.spatial.distance import squareform


def nn_chain_merges(D):
    """(heights, pair counts) of the average-linkage tree of the square
    distances D, by the chain as the kernel runs it."""
    D = D.copy()
    p = D.shape[0]
    size = np.ones(p, dtype=np.int64)
    chain = []
    heights, npairs = [], []
    for _ in range(p - 1):
        if not chain:
            chain.append(int(np.flatnonzero(size > 0)[0]))
        while True:
            x = chain[-1]
            prev = chain[-2] if len(chain) > 1 else -1
            best_v, best_i = np.inf, -1
            for i in range(p):
                if i != x and size[i] > 0 and D[x, i] < best_v:
                    best_v, best_i = D[x, i], i
            if prev >= 0 and not (best_v < D[x, prev]):
                y, cur = prev, D[x, prev]
                break
            chain.append(best_i)
        chain = chain[:-2]
        a, b = min(x, y), max(x, y)
        na, nb = size[a], size[b]
        for i in range(p):
            if i in (a, b) or size[i] == 0:
                continue
            d = (float(na) * D[a, i] + float(nb) * D[b, i]) / float(na + nb)
            D[b, i] = D[i, b] = d
        heights.append(cur)
        npairs.append(float(na) * float(nb))
        size[a] = 0
        size[b] = na + nb
    return np.array(heights), np.array(npairs)


def cophenetic_from_merges(D, heights, npairs):
    p = D.shape[0]
    iu = np.triu_indices(p, 1)
    d = D[iu]
    N = d.size
    md = d.sum() / N
    var_d = ((d - md) ** 2).sum()
    mc = (npairs * heights).sum() / N
    cov = (npairs * (heights - mc) * (heights - md)).sum()
    var_c = (npairs * (heights - mc) ** 2).sum()
    return cov / np.sqrt(var_d * var_c) if var_d > 0 and var_c > 0 else 1.0


def consensus(p, runs, k, seed, noise):
    gen = np.random.default_rng(seed)
    truth = gen.integers(0, k, p)
    C = np.zeros((p, p))
    for _ in range(runs):
        lab = np.where(gen.random(p) < noise, gen.integers(0, k, p), truth)
        C += lab[:, None] == lab[None, :]
    return (C / runs).astype(np.float32)


@pytest.mark.parametrize("p,runs,k,seed,noise", [(40, 8, 3, 0, 0.3), (90, 16, 5, 1, 0.5),
                                                 (120, 64, 4, 2, 0.2), (75, 4, 6, 3, 0.6)])
def test_merges_formula_matches_scipy(p, runs, k, seed, noise):
    C = consensus(p, runs, k, seed, noise).astype(np.float64)
    np.fill_diagonal(C, 1.0)
    D = 1.0 - C
    cond = squareform(D, checks=False)
    c_ref, _ = cophenet(linkage(cond, method="average"), cond)
    h, n = nn_chain_merges(D)
    assert abs(cophenetic_from_merges(D, h, n) - c_ref) <= 1e-12
    # the heights are scipy's merge heights (as a multiset)
    Z = linkage(cond, method="average")
    np.testing.assert_allclose(np.sort(h), np.sort(Z[:, 2]), rtol=0, atol=1e-15)
