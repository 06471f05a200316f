"""Ranks above 32 (the streaming passes' largest bucket) on the GPU against
the oracle, which has no rank limit, like the reference (lib.rs:1589
onward).  The wide loop runs the V contractions as FP64 streaming passes over
32-rank chunks and the rest with the rank as a run-time value.

Bounds, written per check (the plain method's): max|dX| / max|X| <= 1e-10
for W and H, relative objective <= 1e-12 (plus the evaluation's rounding
floor); hals / dnmf from NNDSVD starts, held to max(those bounds, 100 x the
oracle's own one-ulp sensitivity) as the dense parity tests hold them."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import rel, rel_max

import nmf_rs
from nmf_rs import _native, synthetic

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-10
OBJ_TOL = 1e-12
EPS = float(np.finfo(np.float64).eps)


def _objective(oracle, method, V, W, H):
    if method == "brunet":
        return oracle.kl_divergence(V, W, H)
    return oracle.euclidean_distance(V, W, H)


def _rel_obj(method, V, a, b):
    scale = float(V.sum()) if method == "brunet" else 0.5 * float((V * V).sum())
    return max(0.0, abs(a - b) - 10 * EPS * scale) / max(abs(b), 1e-300)


def _sensitivity(oracle, method, V, W0, H0, iters, **kw):
    """How far the oracle's own result moves when W0 is perturbed by one ulp
    (factor measure, objective measure): the HALS sweeps divide by
    max(G_kk, eps), so a component that collapses amplifies rounding."""
    a = oracle.nmf_method(method, V, W0, H0, iters, **kw)
    signs = np.random.default_rng(0).choice([-1.0, 1.0], W0.shape)
    b = oracle.nmf_method(method, V, W0 * (1 + EPS * signs), H0, iters, **kw)
    f = max(rel_max(b["W"], a["W"]), rel_max(b["H"], a["H"]))
    o = _rel_obj(method, V, _objective(oracle, method, V, b["W"], b["H"]),
                 _objective(oracle, method, V, a["W"], a["H"]))
    return f, o


def _check(oracle, method, V, W0, H0, iters, **kw):
    ref = oracle.nmf_method(method, V, W0, H0, iters, **kw)
    got = nmf_rs.nmf(V, W0.shape[1], method, W0=W0, H0=H0, max_iter=iters, **kw)
    tol_f, tol_o = FACTOR_TOL, OBJ_TOL
    if method in ("hals", "dnmf"):
        # max(plain tolerance, 100 x the oracle's one-ulp sensitivity), as the
        # dense parity tests hold the HALS family.
        sf, so = _sensitivity(oracle, method, V, W0, H0, iters, **kw)
        tol_f, tol_o = max(tol_f, 100 * sf), max(tol_o, 100 * so)
    assert got.n_iter == ref["n_iter"]
    dW, dH = rel_max(got.W, ref["W"]), rel_max(got.H, ref["H"])
    assert dW <= tol_f, (dW, tol_f)
    assert dH <= tol_f, (dH, tol_f)
    d_obj = _rel_obj(method, V, _objective(oracle, method, V, got.W, got.H),
                     _objective(oracle, method, V, ref["W"], ref["H"]))
    assert d_obj <= tol_o, (d_obj, tol_o)
    return got, ref


@pytest.mark.parametrize("rank", [33, 48, 64, 100])
@pytest.mark.parametrize("method", ["lee", "brunet"])
def test_wide_rank_mu(oracle, method, rank):
    V = synthetic.counts_matrix(300, 420, 12, 0.3, seed=rank)
    W0, H0 = nmf_rs.random_init(V, rank, seed=rank)
    _check(oracle, method, V, W0, H0, 25)


@pytest.mark.parametrize("rank", [33, 64])
@pytest.mark.parametrize("method", ["hals", "dnmf"])
def test_wide_rank_hals_family(oracle, method, rank):
    # ground-truth rank 48: rank 33 is below it (well conditioned), rank 64
    # above it (surplus components; held to the sensitivity bound)
    V = synthetic.counts_matrix(400, 500, 48, 0.3, seed=rank + 1)
    W0, H0 = nmf_rs.nndsvd_init(V, rank, fill="mean", seed=0)
    _check(oracle, method, V, W0, H0, 20)


@pytest.mark.parametrize("method", ["lee", "brunet"])
def test_wide_rank_stationary(oracle, method):
    V = synthetic.counts_matrix(200, 260, 8, 0.3, seed=4)
    W0, H0 = nmf_rs.random_init(V, 40, seed=4)
    kw = dict(stop="stationary", stationary_th=1e-3, check_interval=5, check_niter=4)
    got, ref = _check(oracle, method, V, W0, H0, 120, **kw)
    assert got.deviances.size == len(ref["deviances"]) == got.n_iter + 1
    assert max(rel(a, b) for a, b in zip(got.deviances, ref["deviances"])) <= OBJ_TOL


def test_wide_rank_ragged_and_device_entry(oracle):
    """Ragged shapes (one row / column short of the tiles) and the device
    entry on an unpadded V (copied to a pitched buffer inside)."""
    import torch

    V = synthetic.counts_matrix(129, 67, 6, 0.3, seed=2)
    W0, H0 = nmf_rs.random_init(V, 37, seed=1)
    ref = oracle.nmf_method("lee", V, W0, H0, 15)
    dV = torch.from_numpy(V).cuda()
    dW = torch.from_numpy(W0.copy()).cuda()
    dH = torch.from_numpy(H0.copy()).cuda()
    ctx = _native.Context(0)
    o = _native.default_options()
    o.method = _native.parse_method("lee")
    o.max_iter = 15
    ctx.run(o, 129, 67, 37, dV.data_ptr(), _native.F64, 67, dW.data_ptr(), dH.data_ptr())
    ctx.close()
    assert rel_max(dW.cpu().numpy(), ref["W"]) <= FACTOR_TOL
    assert rel_max(dH.cpu().numpy(), ref["H"]) <= FACTOR_TOL
