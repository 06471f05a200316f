"""The CPU oracle pinned against the reference's own recorded outputs
(examples/tutorial_quickstart.ipynb) and its Rust unit test
(rust/src/lib.rs:2208-2227).  CPU only."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import rel, rel_max

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import make_golden  # noqa: E402


def test_fixture_inputs_regenerate(quickstart, kats):
    V, W0, H0 = quickstart
    V2, W02, H02 = make_golden.quickstart_inputs()
    np.testing.assert_array_equal(V, V2)
    np.testing.assert_array_equal(W0, W02)
    np.testing.assert_array_equal(H0, H02)
    assert V.min() == kats["V_min"] and V.max() == kats["V_max"]


def test_brunet_200_norm(oracle, quickstart, kats):
    V, W0, H0 = quickstart
    res = oracle.nmf_run("brunet", V, W0, H0, 200)
    norm = float(np.linalg.norm(V - res["W"] @ res["H"]))
    assert rel(norm, kats["brunet_200_frob_norm"]) < 1e-13
    assert res["n_iter"] == 200 and res["deviances"].size == 0


def test_lee_200_norm(oracle, quickstart, kats):
    V, W0, H0 = quickstart
    res = oracle.nmf_run("lee", V, W0, H0, 200)
    norm = float(np.linalg.norm(V - res["W"] @ res["H"]))
    assert round(norm, 4) == kats["lee_200_frob_norm_4dp"]


def test_offset_200_kat(oracle, quickstart, kats):
    # The notebook prints ||V - fitted()|| with fitted() = W H + offset.
    V, W0, H0 = quickstart
    res = oracle.nmf_method("offset", V, W0, H0, 200)
    fitted = res["W"] @ res["H"] + res["offset"][:, None]
    assert round(float(np.linalg.norm(V - fitted)), 4) == kats["offset_200_frob_norm_4dp"]
    lo, hi = kats["offset_200_range_2dp"]
    assert round(float(res["offset"].min()), 2) == lo
    assert round(float(res["offset"].max()), 2) == hi


def test_nsnmf_200_kat(oracle, quickstart, kats):
    # fitted() is W H for nsNMF (no smoothing matrix).
    V, W0, H0 = quickstart
    res = oracle.nmf_method("nsNMF", V, W0, H0, 200)
    assert round(float(np.linalg.norm(V - res["W"] @ res["H"])), 4) == \
        kats["nsnmf_200_frob_norm_4dp"]


def test_offset_default_is_row_means(oracle, quickstart):
    V, W0, H0 = quickstart
    a = oracle.nmf_offset(V, W0, H0, 5)
    b = oracle.nmf_offset(V, W0, H0, 5, offset=np.cumsum(V, axis=1)[:, -1] / V.shape[1])
    np.testing.assert_array_equal(a["W"], b["W"])
    np.testing.assert_array_equal(a["offset"], b["offset"])


def test_offset_nsnmf_stationary_deviances(oracle, quickstart):
    V, W0, H0 = quickstart
    res = oracle.nmf_offset(V, W0, H0, 20, stop="stationary", check_interval=5, check_niter=2)
    d = res["deviances"]
    assert d.size == res["n_iter"] + 1
    assert d[-1] == oracle.euclidean_distance_offset(V, res["W"], res["H"], res["offset"])
    assert np.all(np.diff(d) <= 1e-9 * d[0])  # the offset updates do not raise the loss
    res = oracle.nmf_nsnmf(V, W0, H0, 20, stop="stationary", check_interval=5, check_niter=2)
    S = np.full((5, 5), 0.1) + 0.5 * np.eye(5)
    assert res["deviances"].size == res["n_iter"] + 1
    assert rel(res["deviances"][-1], oracle.kl_divergence(V, res["W"] @ S, res["H"])) < 1e-12


def test_brunet_stationary_kat(oracle, quickstart, kats):
    V, W0, H0 = quickstart
    k = kats["brunet_stationary"]
    res = oracle.nmf_run("brunet", V, W0, H0, k["max_iter"], stop="stationary",
                         stationary_th=k["stationary_th"], check_interval=k["check_interval"],
                         check_niter=k["check_niter"])
    assert res["n_iter"] == k["n_iter"]
    assert res["deviances"].size == k["n_deviances"]
    # The KL sum is one sequential reduction in a fixed order: bit-exact.
    assert res["deviances"][-1] == k["final_kl"]


def test_single_step_delta_kl(oracle, quickstart, kats):
    V, W0, H0 = quickstart
    H1 = oracle.update_h_brunet(V, W0, H0)
    W1 = oracle.update_w_brunet(V, W0, H1)

    def kl(W, H):  # the notebook's own expression (cell 13)
        WH = W @ H
        return float((V * np.log(np.where(V > 0, V / (WH + 1e-30), 1)) - V + WH).sum())

    assert rel(kl(W0, H0) - kl(W1, H1), kats["single_step_brunet_delta_kl"]) < 1e-13


@pytest.mark.parametrize("method", ["brunet", "lee", "offset", "nsNMF", "hals", "ehals",
                                    "dnmf"])
def test_thread_count_independent(oracle, quickstart, method):
    V, W0, H0 = quickstart
    a = oracle.nmf_method(method, V, W0, H0, 30, num_threads=1)
    b = oracle.nmf_method(method, V, W0, H0, 30, num_threads=4)
    np.testing.assert_array_equal(a["W"], b["W"])
    np.testing.assert_array_equal(a["H"], b["H"])


def test_rust_unit_brunet_reduces_kl(oracle):
    # lib.rs:2208-2227: 3x2 V, W0 = 0.5, H0 = 1, brunet 50 it, stationary.
    V = np.array([[1.0, 2.0], [3.0, 4.0], [5.0, 6.0]])
    W0 = np.full((3, 2), 0.5)
    H0 = np.ones((2, 2))
    res = oracle.nmf_run("brunet", V, W0, H0, 50, stop="stationary", stationary_th=1e-12,
                         check_interval=50, check_niter=10)
    assert (res["W"] >= 0).all() and (res["H"] >= 0).all()
    assert res["deviances"][-1] <= res["deviances"][0]


def test_check_interval_zero_mirrors_panic(oracle, quickstart):
    V, W0, H0 = quickstart
    # With a window of 1 sample, the first window closes at iteration 1, the
    # criterion fails (th = 0), the window resets and iteration 2 evaluates
    # `2 % 0` -- the point where the reference panics.
    with pytest.raises(ZeroDivisionError):
        oracle.nmf_run("lee", V, W0, H0, 5, stop="stationary", stationary_th=0.0,
                       check_interval=0, check_niter=1)


@pytest.mark.parametrize("method", ["hals", "ehals", "dnmf"])
def test_hals_family_decreases_loss(oracle, quickstart, method):
    V, W0, H0 = quickstart
    res = oracle.nmf_method(method, V, W0, H0, 50, stop="stationary", check_interval=10)
    dev = res["deviances"]
    assert dev[-1] < dev[0]
    assert (res["W"] > 0).all() and (res["H"] > 0).all()


def test_dnmf_unit_norm_columns(oracle, quickstart):
    V, W0, H0 = quickstart
    res = oracle.nmf_method("dnmf", V, W0, H0, 20)
    norms = np.linalg.norm(res["W"], axis=0)
    np.testing.assert_allclose(norms, 1.0, rtol=1e-12)


def test_ehals_is_hals_from_the_extrapolated_point(oracle, quickstart):
    # One ehals iteration from (W0, H0) with no history is max(eps, .) of the
    # start followed by a HALS sweep (lib.rs:743-776).
    V, W0, H0 = quickstart
    W0 = W0.copy()
    W0[0, 0] = 0.0  # raised to eps by the extrapolation
    a = oracle.nmf_method("ehals", V, W0, H0, 1)
    b = oracle.nmf_method("hals", V, np.maximum(W0, 1e-9), np.maximum(H0, 1e-9), 1)
    np.testing.assert_array_equal(a["W"], b["W"])
    np.testing.assert_array_equal(a["H"], b["H"])
    # Two iterations differ from HALS: the second extrapolates.
    a2 = oracle.nmf_method("ehals", V, W0, H0, 2)
    b2 = oracle.nmf_method("hals", V, np.maximum(W0, 1e-9), np.maximum(H0, 1e-9), 2)
    assert not np.array_equal(a2["W"], b2["W"])


def test_lsnmf_unit_weights_is_lee_without_rescale(oracle, quickstart):
    # W^T((W H) o 1) = W^T W H and ((W H) o 1) H^T = W H H^T: lee's updates
    # (lib.rs:990-1018 vs 213-322) up to summation order; lee's W clamp
    # differs only for NaN.
    V, W0, H0 = quickstart
    a = oracle.nmf_method("lsnmf", V, W0, H0, 50, weight=np.ones_like(V))
    b = oracle.nmf_method("lee", V, W0, H0, 50, rescale=False)
    assert rel_max(a["W"], b["W"]) < 1e-12 and rel_max(a["H"], b["H"]) < 1e-12


def test_lsnmf_ignores_zero_weight_entries(oracle, quickstart):
    V, W0, H0 = quickstart
    gen = np.random.default_rng(3)
    S = (gen.random(V.shape) > 0.1).astype(float)
    V2 = V.copy()
    V2[S == 0] = 1e3  # held-out entries may hold anything
    a = oracle.nmf_method("lsnmf", V, W0, H0, 20, weight=S)
    b = oracle.nmf_method("lsnmf", V2, W0, H0, 20, weight=S)
    np.testing.assert_array_equal(a["W"], b["W"])
    np.testing.assert_array_equal(a["H"], b["H"])


def test_lsnmf_stationary_trace(oracle, quickstart):
    V, W0, H0 = quickstart
    S = np.random.default_rng(5).uniform(0.2, 1.5, V.shape)
    res = oracle.nmf_method("lsnmf", V, W0, H0, 30, weight=S, stop="stationary",
                            check_interval=5, check_niter=2)
    d = res["deviances"]
    assert d.size == res["n_iter"] + 1
    assert d[-1] == oracle.weighted_distance(V, S, res["W"], res["H"])
    assert d[-1] < d[0]
    with pytest.raises(ValueError, match="weight"):
        oracle.nmf_method("lsnmf", V, W0, H0, 3)


# ---------------------------------------------------------------------------
# Kim-Park snmf/r, snmf/l (FCNNLS): the reference's own unit tests of its
# FCNNLS (rust/src/fcnnls.rs tests) and behavioural tests
# (tests/test_lsnmf_snmf.py), on the restatement.
# ---------------------------------------------------------------------------

def test_fcnnls_cholesky_identity(oracle):
    ok, L = oracle.cholesky(np.array([[4.0, 12.0, -16.0], [12.0, 37.0, -43.0],
                                      [-16.0, -43.0, 98.0]]))
    assert ok
    np.testing.assert_allclose(L, [[2, 0, 0], [6, 1, 0], [-8, 5, 3]], atol=1e-12)


def test_fcnnls_unconstrained_active(oracle):
    x = np.array([[1.0, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [0, 1, 1]])
    y = np.array([[2.0, 1.0], [3.0, 2.0], [4.0, 3.0], [4.5, 2.5], [6.5, 4.5]])
    K = oracle.fcnnls(x.T @ x, x.T @ y, eps=0.0)
    assert (K >= -1e-9).all()
    assert ((x @ K - y) ** 2).sum() < 1.0


def test_fcnnls_matches_scipy_nnls_when_well_posed(oracle):
    from scipy.optimize import nnls

    gen = np.random.default_rng(4)
    x = gen.uniform(0, 1, (40, 6))
    y = gen.uniform(-0.5, 1.5, (40, 25))
    K = oracle.fcnnls(x.T @ x, x.T @ y, eps=0.0)
    for j in range(y.shape[1]):
        ref, _ = nnls(x, y[:, j])
        assert np.abs(K[:, j] - ref).max() <= 1e-8


@pytest.fixture(scope="module")
def synth():
    rng = np.random.default_rng(42)
    n, p, rank = 120, 60, 6
    V = rng.uniform(0.1, 1.5, (n, rank)) @ rng.uniform(0.1, 1.5, (rank, p)) + \
        rng.uniform(0, 0.05, (n, p))
    gen = np.random.default_rng(0)
    W0 = gen.uniform(0, V.max(), (n, rank))
    H0 = gen.uniform(0, V.max(), (rank, p))
    return V, W0, H0


@pytest.mark.parametrize("left", [False, True])
def test_snmf_sparser_than_lee(oracle, synth, left):
    V, W0, H0 = synth
    lee = oracle.nmf_method("lee", V, W0, H0, 200)
    res = oracle.nmf_method("snmf/l" if left else "snmf/r", V, W0, H0, 20, sparsity=0.5,
                            smoothness=-1.0)
    dens = lambda M: float((M > 1e-6).mean())  # noqa: E731
    if left:
        assert dens(res["W"]) < dens(lee["W"])
    else:
        assert dens(res["H"]) < dens(lee["H"])
    assert res["n_iter"] == 20 and res["deviances"].size == 20
    assert np.isfinite(res["W"]).all() and np.isfinite(res["H"]).all()


def test_snmf_thread_count_independent(oracle, synth):
    V, W0, H0 = synth
    a = oracle.nmf_method("snmf/r", V, W0, H0, 5, sparsity=0.5, smoothness=-1.0, num_threads=1)
    b = oracle.nmf_method("snmf/r", V, W0, H0, 5, sparsity=0.5, smoothness=-1.0, num_threads=4)
    np.testing.assert_array_equal(a["W"], b["W"])
    np.testing.assert_array_equal(a["H"], b["H"])
