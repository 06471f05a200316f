"""The reference's own behavioural tests of the methods this engine builds
(tests/test_lsnmf_snmf.py of omicverse/rust-NMF: the lsNMF and alias checks),
restated on the GPU path with the same inputs and thresholds.""" 
from __future__ import annotations

import numpy as np
import pytest

import nmf_rs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def synth():
    rng = np.random.default_rng(42)
    n, p, rank = 120, 60, 6
    W_true = rng.uniform(0.1, 1.5, (n, rank))
    H_true = rng.uniform(0.1, 1.5, (rank, p))
    V = W_true @ H_true + rng.uniform(0, 0.05, (n, p))
    W0, H0 = nmf_rs.random_init(V, rank, seed=0)
    return {"V": V, "W0": W0, "H0": H0, "rank": rank}


def test_lsnmf_uniform_weight_close_to_lee(synth):
    V, W0, H0, rank = synth["V"], synth["W0"], synth["H0"], synth["rank"]
    res_ls = nmf_rs.nmf(V, rank=rank, method="lsnmf", weight=np.ones_like(V), W0=W0, H0=H0,
                        max_iter=200, num_threads=2)
    res_lee = nmf_rs.nmf(V, rank=rank, method="lee", W0=W0, H0=H0, max_iter=200,
                         num_threads=2)
    err_ls = np.linalg.norm(V - res_ls.fitted())
    err_lee = np.linalg.norm(V - res_lee.fitted())
    assert err_lee * 0.95 < err_ls < err_lee * 1.05


def test_lsnmf_masking_drops_entries(synth):
    V, W0, H0, rank = synth["V"], synth["W0"], synth["H0"], synth["rank"]
    mask = np.random.default_rng(7).random(V.shape) > 0.20
    V_masked = V.copy()
    V_masked[~mask] = 0
    res = nmf_rs.nmf(V_masked, rank=rank, method="lsnmf", weight=mask.astype(np.float64),
                     W0=W0, H0=H0, max_iter=200, num_threads=2)
    fit = res.fitted()
    assert np.sqrt(((V[mask] - fit[mask]) ** 2).mean()) < 0.3


def test_lsnmf_requires_weight(synth):
    V, W0, H0, rank = synth["V"], synth["W0"], synth["H0"], synth["rank"]
    with pytest.raises((ValueError, RuntimeError)):
        nmf_rs.nmf(V, rank=rank, method="lsnmf", W0=W0, H0=H0, max_iter=10, num_threads=1)


@pytest.mark.parametrize("method,which", [("snmf/r", "H"), ("snmf/l", "W")])
def test_snmf_makes_the_factor_sparser(synth, method, which):
    V, W0, H0, rank = synth["V"], synth["W0"], synth["H0"], synth["rank"]
    res_lee = nmf_rs.nmf(V, rank=rank, method="lee", W0=W0, H0=H0, max_iter=200, num_threads=2)
    res_s = nmf_rs.nmf(V, rank=rank, method=method, sparsity=0.5, smoothness=-1.0, W0=W0,
                       H0=H0, max_iter=20, num_threads=2)
    dens = lambda M: float((M > 1e-6).mean())  # noqa: E731
    assert dens(getattr(res_s, which)) < dens(getattr(res_lee, which))


def test_method_aliases():
    V = np.abs(np.random.default_rng(0).normal(size=(40, 20)))
    W0, H0 = nmf_rs.random_init(V, 3, seed=0)
    pairs = [("ls-nmf", "lsnmf"), ("kl", "brunet"), ("frobenius", "lee"), ("euclidean", "lee"),
             ("ns", "nsnmf"), ("ns_nmf", "nsNMF"), ("e-hals", "ehals"), ("extrap_hals", "ehals"),
             ("diag_nmf", "dnmf"), ("rcppml", "dnmf"), ("snmf_r", "snmf/r"),
             ("snmf_l", "snmf/l")]
    for a, b in pairs:
        kw = dict(W0=W0, H0=H0, max_iter=20, num_threads=1)
        if b == "lsnmf":
            kw["weight"] = np.ones_like(V)
        ra = nmf_rs.nmf(V, rank=3, method=a, **kw)
        rb = nmf_rs.nmf(V, rank=3, method=b, **kw)
        np.testing.assert_array_equal(ra.W, rb.W, err_msg=f"{a} vs {b}")
        np.testing.assert_array_equal(ra.H, rb.H, err_msg=f"{a} vs {b}")
