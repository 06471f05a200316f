"""The split-bf16 precision form (tensor-core passes) against the FP64 oracle.

V is held as bf16 hi + lo (about 2^-17 relative), the factors as three bf16
terms; products run on the tensor cores with f32 sums of at most 2048 terms,
everything else in f64, and the last 2 iterations in f64.  Bounds, written
per check: one iteration without refinement within ONE_ITER_TOL = 5e-6
(max|dX| / max|X|) of the oracle -- the split keeps every product down to
about 2^-24 and the ratio to 2^-17, and the largest error measured over these
shapes is 1.3e-6, so a dropped term (a missing Vl Fm product is ~2^-16 =
1.5e-5) or a layout mistake fails; 40 iterations with refinement within 1e-5
relative objective, as the FP32 form."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel, rel_max

import nmf_rs
from nmf_rs import synthetic

pytestmark = pytest.mark.gpu

ONE_ITER_TOL = 5e-6


def _objective(oracle, method, V, W, H):
    if method == "brunet":
        return oracle.kl_divergence(V, W, H)
    return oracle.euclidean_distance(V, W, H)


@pytest.mark.parametrize("n,p,r", [(1000, 1500, 20), (257, 3001, 3), (2000, 700, 32),
                                   (130, 200, 16), (64, 64, 1)])
def test_one_iteration_matches_oracle(oracle, n, p, r):
    V = synthetic.counts_matrix(n, p, max(2, r // 2), 0.3, seed=n + p)
    W0, H0 = nmf_rs.random_init(V, r, seed=3)
    ref = oracle.nmf_method("lee", V, W0, H0, 1)
    got = nmf_rs.nmf(V, r, "lee", W0=W0, H0=H0, max_iter=1, precision="bf16x3",
                     refine_iters=0)
    assert rel_max(got.H, ref["H"]) <= ONE_ITER_TOL, rel_max(got.H, ref["H"])
    assert rel_max(got.W, ref["W"]) <= ONE_ITER_TOL, rel_max(got.W, ref["W"])


# brunet's split-bf16 passes (tcr.cuh): W H and the contraction on the tensor
# cores, the ratio in f32.  Shapes with ragged tiles (128 outputs), chunks
# (64 elements) and segments (2048 terms), ranks 1..32; the two flat shapes
# give a CTA several short tiles in a row (the tile operand is reloaded in
# tensor memory each time).
@pytest.mark.parametrize("n,p,r", [(1000, 1500, 20), (257, 3001, 3), (2000, 700, 32),
                                   (130, 200, 16), (64, 64, 1), (4100, 129, 7),
                                   (100, 40000, 12), (40000, 100, 12)])
def test_brunet_one_iteration_matches_oracle(oracle, n, p, r):
    V = synthetic.counts_matrix(n, p, max(2, r // 2), 0.3, seed=n + p)
    W0, H0 = nmf_rs.random_init(V, r, seed=3)
    ref = oracle.nmf_method("brunet", V, W0, H0, 1)
    got = nmf_rs.nmf(V, r, "brunet", W0=W0, H0=H0, max_iter=1, precision="bf16x3",
                     refine_iters=0)
    assert rel_max(got.H, ref["H"]) <= ONE_ITER_TOL, rel_max(got.H, ref["H"])
    assert rel_max(got.W, ref["W"]) <= ONE_ITER_TOL, rel_max(got.W, ref["W"])


# nsNMF's split-bf16 form runs the same passes on W S (H pass) and S H (W pass);
# rank 24 takes the 192-wide concatenated layouts.
@pytest.mark.parametrize("n,p,r", [(700, 900, 8), (257, 1301, 3), (600, 1100, 24)])
def test_nsnmf_one_iteration_matches_oracle(oracle, n, p, r):
    V = synthetic.counts_matrix(n, p, max(2, r // 2), 0.3, seed=n + p) + 0.01
    W0, H0 = nmf_rs.random_init(V, r, seed=3)
    ref = oracle.nmf_method("nsNMF", V, W0, H0, 1)
    got = nmf_rs.nmf(V, r, "nsNMF", W0=W0, H0=H0, max_iter=1, precision="bf16x3",
                     refine_iters=0)
    assert rel_max(got.H, ref["H"]) <= ONE_ITER_TOL, rel_max(got.H, ref["H"])
    assert rel_max(got.W, ref["W"]) <= ONE_ITER_TOL, rel_max(got.W, ref["W"])


@pytest.mark.parametrize("method", ["lee", "hals", "ehals", "dnmf", "brunet"])
def test_split_bf16_form(oracle, method):
    V, W0, H0 = synthetic.make(synthetic.PBMC_SUBSET)
    if method in ("hals", "ehals"):  # ill conditioned from a random start
        W0, H0 = nmf_rs.nndsvd_init(V, 8, fill="mean", seed=0)
    ref = oracle.nmf_method(method, V, W0, H0, 40)
    got = nmf_rs.nmf(V, 8, method, W0=W0, H0=H0, max_iter=40, precision="bf16x3")
    o_ref = _objective(oracle, method, V, ref["W"], ref["H"])
    o_got = _objective(oracle, method, V, got.W, got.H)
    assert rel(o_got, o_ref) <= 1e-5, rel(o_got, o_ref)


# Many iterations through the rank > 21 variant of the tensor-core ratio
# passes (192-wide concatenated rows, one segment accumulator).
def test_brunet_split_bf16_rank_26_many_iterations(oracle):
    V = synthetic.counts_matrix(900, 1400, 12, 0.3, seed=5)
    W0, H0 = nmf_rs.random_init(V, 26, seed=6)
    ref = oracle.nmf_method("brunet", V, W0, H0, 40)
    got = nmf_rs.nmf(V, 26, "brunet", W0=W0, H0=H0, max_iter=40, precision="bf16x3")
    o_ref = oracle.kl_divergence(V, ref["W"], ref["H"])
    o_got = oracle.kl_divergence(V, got.W, got.H)
    assert rel(o_got, o_ref) <= 1e-5, rel(o_got, o_ref)


def test_brunet_split_bf16_stationary_and_deterministic():
    # The stationary stop evaluates the objective on the device each
    # iteration, so these iterations are launched one by one.
    V, W0, H0 = synthetic.make(synthetic.PBMC_SUBSET)
    kw = dict(max_iter=60, precision="bf16x3", stop="stationary", check_interval=10,
              check_niter=3, stationary_th=1e-12)
    a = nmf_rs.nmf(V, 8, "brunet", W0=W0, H0=H0, **kw)
    b = nmf_rs.nmf(V, 8, "brunet", W0=W0, H0=H0, **kw)
    np.testing.assert_array_equal(a.W, b.W)
    np.testing.assert_array_equal(a.deviances, b.deviances)
    assert a.deviances.size == a.n_iter + 1


def test_split_bf16_stationary_and_deterministic(oracle):
    V, W0, H0 = synthetic.make(synthetic.PBMC_SUBSET)
    kw = dict(max_iter=60, precision="bf16x3", stop="stationary", check_interval=10,
              check_niter=3, stationary_th=1e-12)
    a = nmf_rs.nmf(V, 8, "lee", W0=W0, H0=H0, **kw)
    b = nmf_rs.nmf(V, 8, "lee", W0=W0, H0=H0, **kw)
    np.testing.assert_array_equal(a.W, b.W)
    np.testing.assert_array_equal(a.deviances, b.deviances)
    assert a.deviances.size == a.n_iter + 1
