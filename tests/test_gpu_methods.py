"""GPU parity of the offset and nsNMF methods (nmf_run_offset, lib.rs:1650-1760;
nmf_run_nsnmf, lib.rs:1762-1830) against the CPU oracle and the reference's
recorded quickstart outputs.

Tolerances (FP64), as for the other methods:
  factors and offsets  max|d| / max|ref| <= 1e-10,
  objective            relative 1e-12 beyond the evaluation's rounding floor.
Reduced precisions (fp32, bf16x3 with their trailing FP64 iterations): the
objective within 1e-5 relative of the FP64 oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel, rel_max

import nmf_rs
from nmf_rs import synthetic

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-10
OBJ_TOL = 1e-12
EPS = float(np.finfo(np.float64).eps)


def _smooth(r, theta):
    return (1.0 - theta) * np.eye(r) + theta / r


def _objective(oracle, method, V, W, H, off=None, theta=0.5):
    if method == "offset":
        return oracle.euclidean_distance_offset(V, W, H, off)
    return oracle.kl_divergence(V, W @ _smooth(W.shape[1], theta), H)


def _rel_obj(method, V, a, b):
    scale = 0.5 * float((V * V).sum()) if method == "offset" else float(V.sum())
    excess = max(0.0, abs(a - b) - 10 * EPS * scale)
    return excess / max(abs(b), 1e-300)


def _check(oracle, method, V, W0, H0, iters, **kw):
    ref = oracle.nmf_method(method, V, W0, H0, iters, **kw)
    got = nmf_rs.nmf(V, W0.shape[1], method, W0=W0, H0=H0, max_iter=iters, **kw)
    assert got.n_iter == ref["n_iter"]
    assert rel_max(got.W, ref["W"]) <= FACTOR_TOL, rel_max(got.W, ref["W"])
    assert rel_max(got.H, ref["H"]) <= FACTOR_TOL, rel_max(got.H, ref["H"])
    if method == "offset":
        assert got.offset is not None and got.offset.shape == (V.shape[0],)
        assert rel_max(got.offset, ref["offset"]) <= FACTOR_TOL
    else:
        assert got.offset is None
    theta = kw.get("theta", 0.5)
    o_got = _objective(oracle, method, V, got.W, got.H, got.offset, theta)
    o_ref = _objective(oracle, method, V, ref["W"], ref["H"], ref.get("offset"), theta)
    assert _rel_obj(method, V, o_got, o_ref) <= OBJ_TOL
    return got, ref


def test_kat_offset_200(quickstart, kats):
    V, W0, H0 = quickstart
    res = nmf_rs.nmf(V, 5, "offset", W0=W0, H0=H0, max_iter=200)
    assert round(float(np.linalg.norm(V - res.fitted())), 4) == kats["offset_200_frob_norm_4dp"]
    lo, hi = kats["offset_200_range_2dp"]
    assert round(float(res.offset.min()), 2) == lo and round(float(res.offset.max()), 2) == hi


def test_kat_nsnmf_200(quickstart, kats):
    V, W0, H0 = quickstart
    res = nmf_rs.nmf(V, 5, "nsNMF", W0=W0, H0=H0, max_iter=200)
    assert round(float(np.linalg.norm(V - res.fitted())), 4) == kats["nsnmf_200_frob_norm_4dp"]


@pytest.mark.parametrize("method", ["offset", "nsNMF"])
def test_quickstart_parity(oracle, quickstart, method):
    V, W0, H0 = quickstart
    _check(oracle, method, V, W0, H0, 100)


@pytest.mark.parametrize("method", ["offset", "nsNMF"])
@pytest.mark.parametrize("shape", [(300, 517, 7), (1, 40, 3), (64, 1, 2), (129, 257, 32)])
def test_ragged_shapes(oracle, method, shape):
    n, p, r = shape
    V = synthetic.counts_matrix(n, p, max(1, r // 2), 0.3, seed=n + p)
    V += 0.01  # keep every row sum positive (the offset update divides by it)
    W0, H0 = nmf_rs.random_init(V, r, seed=3)
    _check(oracle, method, V, W0, H0, 25)


def test_offset_given_start(oracle, quickstart):
    V, W0, H0 = quickstart
    off0 = np.linspace(0.2, 1.3, V.shape[0])
    got, ref = _check(oracle, "offset", V, W0, H0, 30, offset=off0)
    assert not np.array_equal(got.offset, oracle.nmf_offset(V, W0, H0, 30)["offset"])


@pytest.mark.parametrize("theta", [0.0, 0.25, 0.9])
def test_nsnmf_theta(oracle, quickstart, theta):
    V, W0, H0 = quickstart
    _check(oracle, "nsNMF", V, W0, H0, 40, theta=theta)


@pytest.mark.parametrize("method", ["offset", "nsNMF"])
def test_stationary(oracle, quickstart, method):
    V, W0, H0 = quickstart
    kw = dict(stop="stationary", stationary_th=1e-6, check_interval=10, check_niter=5)
    got, ref = _check(oracle, method, V, W0, H0, 300, **kw)
    assert got.deviances.size == ref["deviances"].size == got.n_iter + 1
    d = np.abs(got.deviances - ref["deviances"]) / np.abs(ref["deviances"])
    assert d.max() <= 1e-10, d.max()


@pytest.mark.parametrize("method", ["offset", "nsNMF"])
@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_reduced_precision(oracle, method, precision):
    V = synthetic.counts_matrix(700, 900, 6, 0.3, seed=11) + 0.01
    W0, H0 = nmf_rs.random_init(V, 8, seed=5)
    ref = oracle.nmf_method(method, V, W0, H0, 40)
    got = nmf_rs.nmf(V, 8, method, W0=W0, H0=H0, max_iter=40, precision=precision)
    o_ref = _objective(oracle, method, V, ref["W"], ref["H"], ref.get("offset"))
    o_got = _objective(oracle, method, V, got.W, got.H, got.offset)
    assert rel(o_got, o_ref) <= 1e-5, rel(o_got, o_ref)


def test_offset_through_the_server_and_the_device_entry(oracle):
    """The offset method's row offsets come back from a served request
    (nmfcu_server_submit_offset) and from the device-pointer entry
    (nmfcu_run_offset_device): both equal nmf()'s run bit for bit, and the
    oracle to the plain tolerance."""
    import ctypes

    import torch

    V = synthetic.counts_matrix(140, 230, 3, 0.3, seed=1) + 0.01
    W0, H0 = nmf_rs.random_init(V, 4, seed=1)
    ref = oracle.nmf_method("offset", V, W0, H0, 30)
    alone = nmf_rs.nmf(V, 4, "offset", W0=W0, H0=H0, max_iter=30)
    assert rel_max(alone.offset, ref["offset"]) <= FACTOR_TOL
    off0 = V.mean(axis=1) * 0.5
    given = nmf_rs.nmf(V, 4, "offset", W0=W0, H0=H0, max_iter=30, offset=off0)
    with nmf_rs.serve.Server(slots=2) as srv:
        a = srv.submit(V, 4, "offset", W0=W0, H0=H0, max_iter=30)
        b = srv.submit(V, 4, "offset", W0=W0, H0=H0, max_iter=30, offset=off0)
        c = srv.submit(V, 4, "nsNMF", W0=W0, H0=H0, max_iter=5)
        ra, rb = a.result(timeout=120), b.result(timeout=120)
        assert c.result(timeout=120).offset is None
    for got, want in ((ra, alone), (rb, given)):
        np.testing.assert_array_equal(got.W, want.W)
        np.testing.assert_array_equal(got.H, want.H)
        np.testing.assert_array_equal(got.offset, want.offset)
    # The device entry, V / factors / offsets as device tensors.
    dV = torch.from_numpy(V).cuda()
    dW = torch.from_numpy(W0.copy()).cuda()
    dH = torch.from_numpy(H0.copy()).cuda()
    dO = torch.empty(V.shape[0], dtype=torch.float64, device="cuda")
    o = nmf_rs._native.default_options()
    o.method = nmf_rs._native.parse_method("offset")
    o.max_iter = 30
    ctx = nmf_rs._native.Context(0)
    nd, ni = ctypes.c_int64(0), ctypes.c_int64(0)
    nmf_rs._native.check(nmf_rs._native.load().nmfcu_run_offset_device(
        ctx.handle, ctypes.byref(o), V.shape[0], V.shape[1], 4, ctypes.c_void_p(dV.data_ptr()),
        nmf_rs._native.F64, V.shape[1], None, 0, ctypes.c_void_p(dW.data_ptr()),
        ctypes.c_void_p(dH.data_ptr()), None, ctypes.c_void_p(dO.data_ptr()), None,
        ctypes.byref(nd), ctypes.byref(ni), None))
    ctx.close()
    np.testing.assert_array_equal(dO.cpu().numpy(), alone.offset)
    np.testing.assert_array_equal(dW.cpu().numpy(), alone.W)
    # The plain device entry still refuses offset (it has no slot for them).
    ctx = nmf_rs._native.Context(0)
    with pytest.raises(NotImplementedError, match="nmfcu_run_offset_device"):
        ctx.run(o, V.shape[0], V.shape[1], 4, dV.data_ptr(), nmf_rs._native.F64, V.shape[1],
                dW.data_ptr(), dH.data_ptr())
    ctx.close()


# ---------------------------------------------------------------------------
# lsNMF (nmf_run_lsnmf, lib.rs:945-1043) and cv_rank (__init__.py:273-355)
# ---------------------------------------------------------------------------

def _ls_check(oracle, V, S, W0, H0, iters, **kw):
    ref = oracle.nmf_method("lsnmf", V, W0, H0, iters, weight=S, **kw)
    got = nmf_rs.nmf(V, W0.shape[1], "lsnmf", W0=W0, H0=H0, weight=S, max_iter=iters, **kw)
    assert got.n_iter == ref["n_iter"]
    assert rel_max(got.W, ref["W"]) <= FACTOR_TOL, rel_max(got.W, ref["W"])
    assert rel_max(got.H, ref["H"]) <= FACTOR_TOL, rel_max(got.H, ref["H"])
    o_got = oracle.weighted_distance(V, S, got.W, got.H)
    o_ref = oracle.weighted_distance(V, S, ref["W"], ref["H"])
    assert _rel_obj("offset", V * S, o_got, o_ref) <= OBJ_TOL
    return got, ref


@pytest.mark.parametrize("kind", ["mask", "uniform", "ones"])
def test_lsnmf_quickstart(oracle, quickstart, kind):
    V, W0, H0 = quickstart
    gen = np.random.default_rng(1)
    S = {"mask": (gen.random(V.shape) > 0.05).astype(float),
         "uniform": gen.uniform(0.1, 2.0, V.shape),
         "ones": np.ones_like(V)}[kind]
    _ls_check(oracle, V, S, W0, H0, 60)


@pytest.mark.parametrize("shape", [(300, 517, 7), (1, 40, 3), (64, 1, 2), (129, 257, 32)])
def test_lsnmf_ragged(oracle, shape):
    n, p, r = shape
    V = synthetic.counts_matrix(n, p, max(1, r // 2), 0.3, seed=n * 3 + p)
    S = np.random.default_rng(n + p).uniform(0.0, 1.0, V.shape)
    W0, H0 = nmf_rs.random_init(V, r, seed=4)
    _ls_check(oracle, V, S, W0, H0, 20)


def test_lsnmf_stationary(oracle, quickstart):
    V, W0, H0 = quickstart
    S = (np.random.default_rng(2).random(V.shape) > 0.1).astype(float)
    kw = dict(stop="stationary", stationary_th=1e-6, check_interval=10, check_niter=5)
    got, ref = _ls_check(oracle, V, S, W0, H0, 200, **kw)
    assert got.deviances.size == ref["deviances"].size == got.n_iter + 1
    d = np.abs(got.deviances - ref["deviances"]) / np.abs(ref["deviances"])
    assert d.max() <= 1e-10


def test_lsnmf_arguments(quickstart):
    V, W0, H0 = quickstart
    with pytest.raises(ValueError, match="weight"):
        nmf_rs.nmf(V, 5, "lsnmf", W0=W0, H0=H0, max_iter=2)
    with pytest.raises(NotImplementedError, match="FP64"):
        nmf_rs.nmf(V, 5, "lsnmf", W0=W0, H0=H0, weight=np.ones_like(V), max_iter=2,
                   precision="fp32")


def test_cv_rank_prefers_the_true_rank():
    V = synthetic.counts_matrix(200, 300, 4, 0.3, seed=8) + 0.01
    df = nmf_rs.cv_rank(V, [1, 4], n_folds=2, max_iter=60, seed=1)
    assert list(df.columns) == ["rank", "fold", "train_loss", "test_mse"]
    assert len(df) == 4
    mse = df.groupby("rank")["test_mse"].mean()
    assert mse[4] < mse[1]
    again = nmf_rs.cv_rank(V, [1, 4], n_folds=2, max_iter=60, seed=1)
    np.testing.assert_array_equal(df.to_numpy(), again.to_numpy())


def test_ehals_kat_free_parity_from_nndsvd(oracle, quickstart):
    # ehals has no recorded output in the reference; from an NNDSVD start its
    # HALS sweeps are well conditioned, so the plain tolerance applies.
    V = quickstart[0]
    W0, H0 = nmf_rs.nndsvd_init(V, 5, fill="mean", seed=0)
    ref = oracle.nmf_method("ehals", V, W0, H0, 80)
    got = nmf_rs.nmf(V, 5, "ehals", W0=W0, H0=H0, max_iter=80)
    assert rel_max(got.W, ref["W"]) <= FACTOR_TOL and rel_max(got.H, ref["H"]) <= FACTOR_TOL
