"""GPU parity: the CUDA library (called through the C ABI via nmf_rs) against
the CPU oracle and against the reference's recorded quickstart outputs.

Tolerances (FP64 plain method), written per check below:
  factors   max|dW| / max|W| <= 1e-10 and the same for H,
  objective |dObj| <= 1e-12 |Obj| + 10 eps (sum V or 0.5 ||V||^2); the
            second term is the evaluation's own rounding floor and only
            matters for an exact fit.
The GPU sums in a different order than the reference's scalar loops (and
with FMA), so agreement is to rounding, not bitwise.

hals and dnmf are not always well conditioned: from a random start a HALS
component can collapse to the eps floor, after which the sweep divides by
max(G_kk, eps) = eps and amplifies rounding by ~1e9.  The oracle itself then
moves by up to ~1e-3 when W0 is perturbed by one ulp, and so would the
reference (whose W^T V / V H^T summation order, matrixmultiply's, is not
pinned either).  For those two methods the bound is therefore
max(1e-10, 100 x the oracle's own one-ulp sensitivity),
measured in the test; from NNDSVD starts HALS is well conditioned and is
held to the plain tolerance.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel, rel_max

import nmf_rs
from nmf_rs import _native, synthetic

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-10
OBJ_TOL = 1e-12
METHODS = ["brunet", "lee", "hals", "ehals", "dnmf"]


def _objective(oracle, method, V, W, H):
    if method == "brunet":
        return oracle.kl_divergence(V, W, H)
    return oracle.euclidean_distance(V, W, H)


EPS = float(np.finfo(np.float64).eps)


def _obj_noise(method, V):
    """Absolute rounding floor of an objective evaluation: 10 eps x its scale
    (sum V for KL, whose terms cancel to ~eps v each near a fit; 0.5 ||V||^2
    for Frobenius).  Only matters when the fit is (near) exact."""
    scale = float(V.sum()) if method == "brunet" else 0.5 * float((V * V).sum())
    return 10 * EPS * scale


def _rel_obj(method, V, a, b):
    """Relative objective difference beyond the evaluation's rounding floor:
    the check  |a - b| <= tol |b| + floor  is  _rel_obj <= tol."""
    excess = max(0.0, abs(a - b) - _obj_noise(method, V))
    return excess / max(abs(b), 1e-300)


def _sensitivity(oracle, method, V, W0, H0, iters, **kw):
    """How far the oracle's own result moves when W0 is perturbed by one ulp:
    (factor measure, objective measure)."""
    a = oracle.nmf_method(method, V, W0, H0, iters, **kw)
    signs = np.random.default_rng(0).choice([-1.0, 1.0], W0.shape)
    b = oracle.nmf_method(method, V, W0 * (1 + 2.220446049250313e-16 * signs), H0, iters, **kw)
    f = max(rel_max(b["W"], a["W"]), rel_max(b["H"], a["H"]))
    o = _rel_obj(method, V, _objective(oracle, method, V, b["W"], b["H"]),
                 _objective(oracle, method, V, a["W"], a["H"]))
    return f, o


def _check(oracle, method, V, W0, H0, iters, **kw):
    ref = oracle.nmf_method(method, V, W0, H0, iters, **kw)
    got = nmf_rs.nmf(V, W0.shape[1], method, W0=W0, H0=H0, max_iter=iters, **kw)
    tol_f, tol_o = FACTOR_TOL, OBJ_TOL
    if method in ("hals", "ehals", "dnmf"):
        sf, so = _sensitivity(oracle, method, V, W0, H0, iters, **kw)
        tol_f, tol_o = max(tol_f, 100 * sf), max(tol_o, 100 * so)
    assert got.n_iter == ref["n_iter"]
    dW, dH = rel_max(got.W, ref["W"]), rel_max(got.H, ref["H"])
    assert dW <= tol_f, (dW, tol_f)
    assert dH <= tol_f, (dH, tol_f)
    o_got = _objective(oracle, method, V, got.W, got.H)
    o_ref = _objective(oracle, method, V, ref["W"], ref["H"])
    d_obj = _rel_obj(method, V, o_got, o_ref)
    assert d_obj <= tol_o, (d_obj, tol_o)
    return got, ref


# ---------------------------------------------------------------------------
# The reference's own recorded outputs, through the GPU path.
# ---------------------------------------------------------------------------

def test_kat_brunet_200(quickstart, kats):
    V, W0, H0 = quickstart
    res = nmf_rs.nmf(V, 5, "brunet", W0=W0, H0=H0, max_iter=200)
    norm = float(np.linalg.norm(V - res.fitted()))
    assert rel(norm, kats["brunet_200_frob_norm"]) < 1e-10


def test_kat_lee_200(quickstart, kats):
    V, W0, H0 = quickstart
    res = nmf_rs.nmf(V, 5, "lee", W0=W0, H0=H0, max_iter=200)
    assert round(float(np.linalg.norm(V - res.fitted())), 4) == kats["lee_200_frob_norm_4dp"]


def test_kat_brunet_stationary(quickstart, kats):
    V, W0, H0 = quickstart
    k = kats["brunet_stationary"]
    res = nmf_rs.nmf(V, 5, "brunet", W0=W0, H0=H0, max_iter=k["max_iter"], stop="stationary",
                     stationary_th=k["stationary_th"], check_interval=k["check_interval"],
                     check_niter=k["check_niter"])
    assert res.n_iter == k["n_iter"]
    assert res.deviances.size == k["n_deviances"]
    assert rel(float(res.deviances[-1]), k["final_kl"]) < 1e-10


def test_kat_single_step(quickstart, kats):
    V, W0, H0 = quickstart
    H1 = nmf_rs.update_h_brunet(V, W0, H0)
    W1 = nmf_rs.update_w_brunet(V, W0, H1)

    def kl(W, H):
        WH = W @ H
        return float((V * np.log(np.where(V > 0, V / (WH + 1e-30), 1)) - V + WH).sum())

    assert rel(kl(W0, H0) - kl(W1, H1), kats["single_step_brunet_delta_kl"]) < 1e-10


# ---------------------------------------------------------------------------
# Oracle parity.
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("method", METHODS)
def test_quickstart_parity(oracle, quickstart, method):
    V, W0, H0 = quickstart
    _check(oracle, method, V, W0, H0, 100)


@pytest.mark.parametrize("method", ["hals", "ehals", "dnmf"])
@pytest.mark.parametrize("case", ["quickstart", "pbmc-subset"])
def test_hals_family_from_nndsvd_strict(oracle, quickstart, method, case):
    """From an NNDSVD start the HALS family is well conditioned: plain tolerance."""
    if case == "quickstart":
        V = quickstart[0]
        r = 5
    else:
        V = synthetic.counts_matrix(1500, 3000, 8, 0.3, seed=1)
        r = 8
    W0, H0 = nmf_rs.nndsvd_init(V, r, fill="mean", seed=0)
    ref = oracle.nmf_method(method, V, W0, H0, 50)
    got = nmf_rs.nmf(V, r, method, W0=W0, H0=H0, max_iter=50)
    assert rel_max(got.W, ref["W"]) <= FACTOR_TOL
    assert rel_max(got.H, ref["H"]) <= FACTOR_TOL
    o_got = _objective(oracle, method, V, got.W, got.H)
    o_ref = _objective(oracle, method, V, ref["W"], ref["H"])
    assert rel(o_got, o_ref) <= OBJ_TOL


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("shape", [(97, 131, 3), (33, 1000, 13), (517, 64, 1), (64, 33, 32),
                                   (300, 257, 17), (1, 40, 2), (40, 1, 2)])
def test_ragged_shapes(oracle, method, shape):
    n, p, r = shape
    V = synthetic.counts_matrix(n, p, max(2, r // 2), 0.3, seed=n + p + r)
    W0, H0 = nmf_rs.random_init(V, r, seed=11)
    _check(oracle, method, V, W0, H0, 25)


@pytest.mark.parametrize("rank", [1, 2, 5, 7, 8, 10, 11, 16, 20, 23, 27, 31, 32])
def test_every_rank_bucket(oracle, rank):
    V = synthetic.counts_matrix(150, 220, 6, 0.3, seed=rank)
    W0, H0 = nmf_rs.random_init(V, rank, seed=rank)
    for method in ("lee", "brunet"):
        _check(oracle, method, V, W0, H0, 10)


def test_pbmc_subset_lee_full(oracle):
    """lee on the 1500 x 3000 rank-8 workload, 100 iterations."""
    V, W0, H0 = synthetic.make(synthetic.PBMC_SUBSET)
    _check(oracle, "lee", V, W0, H0, 100)


@pytest.mark.parametrize("method", ["brunet", "hals"])
def test_pbmc8k_shape(oracle, method):
    """brunet and hals on the 2000 x 7750 rank-10 workload at its stated 100
    iterations, from its seeded uniform start."""
    V, W0, H0 = synthetic.make(synthetic.PBMC8K_SHAPE)
    _check(oracle, method, V, W0, H0, 100)


@pytest.mark.parametrize("method", METHODS)
def test_stationary_stop_parity(oracle, quickstart, method):
    V, W0, H0 = quickstart
    if method in ("hals", "ehals"):  # well-conditioned start: the deviances compare
        W0, H0 = nmf_rs.nndsvd_init(V, 5, fill="mean", seed=0)
    kw = dict(stop="stationary", stationary_th=1e-3, check_interval=5, check_niter=4)
    got, ref = _check(oracle, method, V, W0, H0, 300, **kw)
    assert got.deviances.size == ref["deviances"].size == got.n_iter + 1
    assert max(rel(a, b) for a, b in zip(got.deviances, ref["deviances"])) <= OBJ_TOL


def test_stationary_stops_early(oracle, quickstart):
    V, W0, H0 = quickstart
    kw = dict(stop="stationary", stationary_th=1.0, check_interval=10, check_niter=3)
    got, ref = _check(oracle, "lee", V, W0, H0, 2000, **kw)
    assert got.n_iter < 2000


def test_max_iter_zero(quickstart):
    V, W0, H0 = quickstart
    res = nmf_rs.nmf(V, 5, "lee", W0=W0, H0=H0, max_iter=0, stop="stationary")
    np.testing.assert_array_equal(res.W, W0)
    np.testing.assert_array_equal(res.H, H0)
    assert res.n_iter == 0 and res.deviances.size == 1


def test_check_interval_zero_raises(quickstart):
    V, W0, H0 = quickstart
    with pytest.raises(ValueError, match="check_interval"):
        nmf_rs.nmf(V, 5, "lee", W0=W0, H0=H0, max_iter=5, stop="stationary",
                   stationary_th=0.0, check_interval=0, check_niter=1)


@pytest.mark.parametrize("step", ["h_brunet", "w_brunet", "h_lee", "w_lee"])
def test_single_steps(oracle, quickstart, step):
    V, W0, H0 = quickstart
    got = getattr(nmf_rs, "update_" + step)(V, W0, H0)
    ref = getattr(oracle, "update_" + step)(V, W0, H0)
    assert rel_max(got, ref) <= 1e-13


def test_objectives(oracle, quickstart):
    V, W0, H0 = quickstart
    assert rel(_native.divergence(V, W0, H0), oracle.kl_divergence(V, W0, H0)) <= OBJ_TOL
    assert rel(_native.distance(V, W0, H0), oracle.euclidean_distance(V, W0, H0)) <= OBJ_TOL


def test_kl_skips_zero_estimate():
    # kl_divergence adds nothing where v > 0 and wh == 0 (lib.rs:1418-1423)
    # and adds wh where v == 0.
    V = np.array([[1.0, 0.0], [2.0, 3.0]])
    W = np.array([[0.0], [1.0]])
    H = np.array([[1.0, 2.0]])
    expected = (2 * np.log(2 / 1) - 2 + 1) + (3 * np.log(3 / 2) - 3 + 2)
    assert rel(_native.divergence(V, W, H), expected) < 1e-15


@pytest.mark.parametrize("method", METHODS)
def test_deterministic(quickstart, method):
    V, W0, H0 = quickstart
    a = nmf_rs.nmf(V, 5, method, W0=W0, H0=H0, max_iter=20)
    b = nmf_rs.nmf(V, 5, method, W0=W0, H0=H0, max_iter=20)
    np.testing.assert_array_equal(a.W, b.W)
    np.testing.assert_array_equal(a.H, b.H)


@pytest.mark.parametrize("method", ["lee", "brunet", "hals", "ehals", "dnmf"])
def test_fp32_precision_form(oracle, method):
    """V in f32 for the contractions, f64 everywhere else, 2 f64 sweeps:
    objective within 1e-5 (relative) of the FP64 oracle."""
    V, W0, H0 = synthetic.make(synthetic.PBMC_SUBSET)
    if method in ("hals", "ehals"):  # ill conditioned from a random start (see top)
        W0, H0 = nmf_rs.nndsvd_init(V, 8, fill="mean", seed=0)
    ref = oracle.nmf_method(method, V, W0, H0, 40)
    got = nmf_rs.nmf(V, 8, method, W0=W0, H0=H0, max_iter=40, precision="fp32")
    o_ref = _objective(oracle, method, V, ref["W"], ref["H"])
    o_got = _objective(oracle, method, V, got.W, got.H)
    assert rel(o_got, o_ref) <= 1e-5, rel(o_got, o_ref)


def test_unsupported_method_and_rank(quickstart):
    V, W0, H0 = quickstart
    with pytest.raises(NotImplementedError):  # snmf runs in FP64 only
        nmf_rs.nmf(V, 5, "snmf/r", W0=W0, H0=H0, max_iter=2, precision="bf16x3")
    V2 = synthetic.counts_matrix(50, 60, 4, 0.3, seed=1)
    with pytest.raises(NotImplementedError, match="rank 257"):
        nmf_rs.nmf(V2, 257, "lee", max_iter=2, seed=0)


def test_nonfinite_propagates_like_reference(oracle, quickstart):
    # lee's H update maps NaN to eps (`temp > eps ? temp : eps`, lib.rs:240).
    V, W0, H0 = quickstart
    H0 = H0.copy()
    H0[0, 0] = np.nan
    got = nmf_rs.update_h_lee(V, W0, H0)
    ref = oracle.update_h_lee(V, W0, H0)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
    mask = ~np.isnan(ref)
    assert rel_max(got[mask], ref[mask]) <= 1e-13
