"""Batched solves (consensus restarts and rank sweeps) on the GPU.

Every solve of a batch must give what the same solve gives alone: FP64
batches are held to the single-solve bounds against the oracle
(max|dW|/max|W| <= 1e-10, objective within 1e-12 relative plus the
evaluation's rounding floor).  The FP32 batch approximates the FP64 result
and is held to max|dW|/max|W| <= 1e-3 and a relative objective difference
<= 1e-5.  Consensus matrices are exact counts and are compared with numpy's
connectivity average to float32 rounding.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_max

import nmf_rs
from nmf_rs import _native, consensus, synthetic

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-10
OBJ_TOL = 1e-12
EPS = float(np.finfo(np.float64).eps)


def _counts(n, p, seed):
    return synthetic.counts_matrix(n, p, 6, 0.3, seed)


def _starts(V, ranks, seed):
    gen = np.random.default_rng(seed)
    out = []
    for r in ranks:
        s = float(np.sqrt(V.mean() / r))
        out.append((gen.uniform(0, s, (V.shape[0], r)), gen.uniform(0, s, (r, V.shape[1]))))
    return out


def _kl_close(oracle, V, W, H, Wr, Hr, tol):
    a = oracle.kl_divergence(V, W, H)
    b = oracle.kl_divergence(V, Wr, Hr)
    floor = 10 * EPS * float(V.sum())
    return max(0.0, abs(a - b) - floor) / abs(b) <= tol, (a, b)


@pytest.mark.parametrize("iters", [0, 7, 37])
def test_batch_fp64_mixed_ranks_match_oracle(oracle, iters):
    V = _counts(300, 700, 11)
    ranks = [1, 2, 3, 3, 5, 7, 8, 16, 16, 4, 12, 9, 10, 11]  # every rank bucket
    starts = _starts(V, ranks, 5)
    got = consensus.run_batch(V, starts, iters, precision="fp64")
    for (W0, H0), (W, H) in zip(starts, got):
        ref = oracle.nmf_method("brunet", V, W0, H0, iters)
        assert rel_max(W, ref["W"]) <= FACTOR_TOL, rel_max(W, ref["W"])
        assert rel_max(H, ref["H"]) <= FACTOR_TOL, rel_max(H, ref["H"])
        ok, vals = _kl_close(oracle, V, W, H, ref["W"], ref["H"], OBJ_TOL)
        assert ok, vals


def test_batch_wide_ranks_match_oracle(oracle):
    """Ranks above the batched kernels' 16 run through the single-solve
    engine in FP64 inside the same call (40 takes the wide loop above 32);
    the rest of the batch is unchanged."""
    V = _counts(200, 300, 21)
    ranks = [3, 17, 5, 20, 40, 2]
    starts = _starts(V, ranks, 6)
    for precision in ("fp64", "fp32"):
        got = consensus.run_batch(V, starts, 12, precision=precision)
        for r, (W0, H0), (W, H) in zip(ranks, starts, got):
            ref = oracle.nmf_method("brunet", V, W0, H0, 12)
            tol = FACTOR_TOL if (precision == "fp64" or r > 16) else 1e-3
            assert rel_max(W, ref["W"]) <= tol, (precision, r, rel_max(W, ref["W"]))
            assert rel_max(H, ref["H"]) <= tol, (precision, r, rel_max(H, ref["H"]))


def test_batch_fp64_many_restarts_one_rank(oracle):
    """23 restarts of rank 3: several CTA groups, the last one padded."""
    V = _counts(257, 513, 3)
    starts = consensus.restart_starts(V, 3, 23)
    got = consensus.run_batch(V, starts, 20, precision="fp64")
    for (W0, H0), (W, H) in zip(starts, got):
        ref = oracle.nmf_method("brunet", V, W0, H0, 20)
        assert rel_max(W, ref["W"]) <= FACTOR_TOL
        assert rel_max(H, ref["H"]) <= FACTOR_TOL


def test_batch_fp32_close_to_fp64(oracle):
    V = _counts(400, 900, 8)
    starts = _starts(V, [2, 5, 10, 10], 9)
    got = consensus.run_batch(V, starts, 30, precision="fp32")
    for (W0, H0), (W, H) in zip(starts, got):
        ref = oracle.nmf_method("brunet", V, W0, H0, 30)
        assert rel_max(W, ref["W"]) <= 1e-3, rel_max(W, ref["W"])
        assert rel_max(H, ref["H"]) <= 1e-3, rel_max(H, ref["H"])
        ok, vals = _kl_close(oracle, V, W, H, ref["W"], ref["H"], 1e-5)
        assert ok, vals


def test_batch_equals_single_solves():
    """Each solve of a batch against the single-solve engine (both FP64)."""
    V = _counts(180, 260, 4)
    starts = consensus.restart_starts(V, 4, 5)
    got = consensus.run_batch(V, starts, 15, precision="fp64")
    for (W0, H0), (W, H) in zip(starts, got):
        one = nmf_rs.nmf(V, 4, "brunet", W0=W0, H0=H0, max_iter=15)
        assert rel_max(W, one.W) <= FACTOR_TOL
        assert rel_max(H, one.H) <= FACTOR_TOL


def _numpy_consensus(Hs):
    acc = np.zeros((Hs[0].shape[1],) * 2)
    for H in Hs:
        acc += consensus.connectivity_matrix(H)
    return acc / len(Hs)


def test_consensus_matrix_matches_numpy():
    gen = np.random.default_rng(1)
    p = 333
    ranks = np.array([3, 5, 3, 7, 3, 2], dtype=np.int32)
    Hs = [gen.random((int(r), p)) for r in ranks]
    dH = torch.from_numpy(np.concatenate(Hs, axis=0)).cuda()
    out = torch.empty((p, p), dtype=torch.float32, device="cuda")
    ctx = _native.Context(0)
    lib = _native.load()
    i32p = ctypes.POINTER(ctypes.c_int32)
    for sel in ([0, 2, 4], [1], [5, 3, 0, 1]):
        s = np.array(sel, dtype=np.int32)
        _native.check(lib.nmfcu_consensus_device(
            ctx.handle, p, len(ranks), ranks.ctypes.data_as(i32p), ctypes.c_void_p(dH.data_ptr()),
            len(s), s.ctypes.data_as(i32p), ctypes.c_void_p(out.data_ptr()),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        want = _numpy_consensus([Hs[i] for i in sel])
        np.testing.assert_allclose(out.cpu().numpy(), want, rtol=0, atol=1e-7)
    ctx.close()


def test_consensus_sweep_batched_equals_one_by_one():
    V = _counts(200, 300, 21)
    kw = dict(ranks=[2, 3], n_runs=4, max_iter=30, precision="fp64")
    a = consensus.consensus_sweep(V, batched=True, **kw)
    b = consensus.consensus_sweep(V, batched=False, **kw)
    assert rel_max(a["W"], b["W"]) <= FACTOR_TOL
    assert rel_max(a["H"], b["H"]) <= FACTOR_TOL
    for k, off in ((2, 0), (3, 8)):
        ca, cb = a["per_rank"][k]["consensus"], b["per_rank"][k]["consensus"]
        np.testing.assert_array_equal(ca, cb)
        Hs = [a["H"][off + i * k: off + (i + 1) * k] for i in range(4)]
        np.testing.assert_allclose(ca, _numpy_consensus(Hs), rtol=0, atol=1e-7)
        assert -1.0 <= a["per_rank"][k]["cophenetic"] <= 1.0
        assert 0.0 <= a["per_rank"][k]["dispersion"] <= 1.0
        host = consensus.cophenetic_correlation(a["per_rank"][k]["consensus"])
        assert a["per_rank"][k]["cophenetic"] == pytest.approx(host, abs=1e-10)


# ---------------------------------------------------------------------------
# Consensus statistics on the device (nmfcu_consensus_stats_device)
# ---------------------------------------------------------------------------

def _tied_consensus(p, runs, k, seed, noise):
    gen = np.random.default_rng(seed)
    truth = gen.integers(0, k, p)
    C = np.zeros((p, p))
    for _ in range(runs):
        lab = np.where(gen.random(p) < noise, gen.integers(0, k, p), truth)
        C += lab[:, None] == lab[None, :]
    return (C / runs).astype(np.float32)


@pytest.mark.parametrize("p,runs,k,seed,noise", [(60, 8, 3, 0, 0.3), (300, 64, 5, 1, 0.4),
                                                 (1500, 64, 6, 2, 0.25), (2, 4, 2, 3, 0.5),
                                                 (1, 4, 2, 4, 0.5)])
def test_consensus_stats_match_scipy(p, runs, k, seed, noise):
    import torch

    from nmf_rs import consensus

    C = _tied_consensus(p, runs, k, seed, noise)
    coph, disp = consensus.consensus_stats(torch.from_numpy(C).cuda())
    assert coph == pytest.approx(consensus.cophenetic_correlation(C), abs=1e-10)
    assert disp == pytest.approx(consensus.dispersion_coefficient(
        np.where(np.eye(p, dtype=bool), 1.0, C.astype(np.float64))), abs=1e-12)


def test_consensus_stats_pitched_input():
    import torch

    from nmf_rs import consensus

    C = _tied_consensus(200, 16, 4, 7, 0.3)
    buf = torch.zeros((200, 256), dtype=torch.float32, device="cuda")
    buf[:, :200] = torch.from_numpy(C)
    a = consensus.consensus_stats(buf[:, :200])
    b = consensus.consensus_stats(torch.from_numpy(C).cuda())
    assert a == b


def test_consensus_stats_batch_equals_one_at_a_time():
    """Several matrices' trees built concurrently (one block each) give the
    same bits as one matrix at a time, and match scipy."""
    import torch

    from nmf_rs import consensus

    mats = [_tied_consensus(700, 32, k, 10 + k, 0.3) for k in (2, 3, 5, 8)]
    stack = torch.from_numpy(np.stack(mats)).cuda()
    got = consensus.consensus_stats_batch(stack)
    for m, C in enumerate(mats):
        assert got[m] == consensus.consensus_stats(torch.from_numpy(C).cuda())
        assert got[m][0] == pytest.approx(consensus.cophenetic_correlation(C), abs=1e-10)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_shapes_agree_and_autotune(precision):
    # The kernel shapes the autotuner picks from regroup solves per CTA; a
    # solve's arithmetic is the same in every shape, so the results agree bit
    # for bit, and the tuned run (which times the shapes on copies of the
    # starting factors) leaves the caller's result unchanged too.
    V = _counts(260, 530, 3)
    ranks = [2, 3, 3, 5, 9, 12, 1, 16]
    starts = _starts(V, ranks, 8)
    got = []
    try:
        for shape in range(consensus.batch_shape_count()):
            consensus.set_batch_shape(shape)
            got.append(consensus.run_batch(V, starts, 24, precision=precision))
            assert consensus.last_batch_shape() == shape
        consensus.set_batch_shape("auto")
        tuned = consensus.run_batch(V, starts, 24, precision=precision)
        assert 0 <= consensus.last_batch_shape() < consensus.batch_shape_count()
    finally:
        consensus.set_batch_shape("auto")
    for other in got[1:] + [tuned]:
        for (W, H), (W2, H2) in zip(got[0], other):
            np.testing.assert_array_equal(W, W2)
            np.testing.assert_array_equal(H, H2)
