"""GPU Kim-Park sparse NMF (snmf/r, snmf/l: nmf_run_snmf_kim_park,
lib.rs:1216-1320 with fcnnls.rs:297-470) against the CPU oracle.

Tolerance: max|dW| / max|W| (and H) <= max(1e-10, 100 x the oracle's own
movement when W0 moves by one ulp): FCNNLS makes discrete active-set
decisions, so where a decision sits near its threshold the reference's own
result is that sensitive to rounding (its normal equations come from
matrixmultiply, whose summation order no test pins).  Deviances: relative
1e-9 or the same bound.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_max

import nmf_rs

pytestmark = pytest.mark.gpu

EPS = 2.220446049250313e-16


@pytest.fixture(scope="module")
def synth():
    rng = np.random.default_rng(42)
    n, p, rank = 120, 60, 6
    V = rng.uniform(0.1, 1.5, (n, rank)) @ rng.uniform(0.1, 1.5, (rank, p)) + \
        rng.uniform(0, 0.05, (n, p))
    W0, H0 = nmf_rs.random_init(V, rank, seed=0)
    return V, W0, H0


def _sensitivity(oracle, method, V, W0, H0, iters, **kw):
    a = oracle.nmf_method(method, V, W0, H0, iters, **kw)
    signs = np.random.default_rng(0).choice([-1.0, 1.0], W0.shape)
    b = oracle.nmf_method(method, V, W0 * (1 + EPS * signs), H0, iters, **kw)
    return a, max(rel_max(b["W"], a["W"]), rel_max(b["H"], a["H"]))


def _check(oracle, method, V, W0, H0, iters, **kw):
    ref, sens = _sensitivity(oracle, method, V, W0, H0, iters, **kw)
    tol = max(1e-10, 100 * sens)
    got = nmf_rs.nmf(V, W0.shape[1], method, W0=W0, H0=H0, max_iter=iters, **kw)
    assert got.n_iter == iters and got.deviances.size == iters
    assert rel_max(got.W, ref["W"]) <= tol, (rel_max(got.W, ref["W"]), tol)
    assert rel_max(got.H, ref["H"]) <= tol, (rel_max(got.H, ref["H"]), tol)
    d = np.abs(got.deviances - ref["deviances"]) / np.abs(ref["deviances"])
    assert d.max() <= max(1e-9, tol), d.max()
    return got, ref


@pytest.mark.parametrize("method", ["snmf/r", "snmf/l"])
def test_snmf_matches_oracle_synth(oracle, synth, method):
    V, W0, H0 = synth
    _check(oracle, method, V, W0, H0, 20, sparsity=0.5, smoothness=-1.0)


@pytest.mark.parametrize("method", ["snmf/r", "snmf/l"])
def test_snmf_matches_oracle_quickstart(oracle, quickstart, method):
    V, W0, H0 = quickstart
    _check(oracle, method, V, W0, H0, 10, sparsity=0.01, smoothness=1.0)


@pytest.mark.parametrize("shape", [(97, 131, 3), (33, 200, 13), (150, 40, 32)])
def test_snmf_ragged(oracle, shape):
    from nmf_rs import synthetic

    n, p, r = shape
    V = synthetic.counts_matrix(n, p, max(2, r // 2), 0.3, seed=n + p) + 0.01
    W0, H0 = nmf_rs.random_init(V, r, seed=3)
    _check(oracle, "snmf/r", V, W0, H0, 6, sparsity=0.1, smoothness=-1.0)


@pytest.mark.parametrize("method,which", [("snmf/r", "H"), ("snmf/l", "W")])
def test_snmf_sparser_than_lee(synth, method, which):
    # the reference's tests/test_lsnmf_snmf.py checks, same inputs and thresholds
    V, W0, H0 = synth
    lee = nmf_rs.nmf(V, rank=6, method="lee", W0=W0, H0=H0, max_iter=200)
    s = nmf_rs.nmf(V, rank=6, method=method, sparsity=0.5, smoothness=-1.0, W0=W0, H0=H0,
                   max_iter=20)
    dens = lambda M: float((M > 1e-6).mean())  # noqa: E731
    assert dens(getattr(s, which)) < dens(getattr(lee, which))


def test_snmf_fp64_only(synth):
    V, W0, H0 = synth
    with pytest.raises(NotImplementedError, match="FP64"):
        nmf_rs.nmf(V, 6, "snmf/r", W0=W0, H0=H0, max_iter=2, precision="fp32")
