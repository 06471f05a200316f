"""Sparse V (CSR) on the GPU against the dense oracle.

The CSR path (nmfcu_run_csr) reads only the stored entries; the oracle runs
the reference's dense loop on the same V densified.  Bounds, written per
check (the plain method's): max|dX| / max|X| <= 1e-10 for W and H, relative
objective <= 1e-12 (plus the evaluation's rounding floor, as the dense
parity tests), deviances of the stationary stop per iteration within 1e-12.
hals / dnmf start from NNDSVD (well conditioned, as in the dense tests)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

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


def _sparsify(V, density, seed):
    """V with all but about `density` of its entries set to zero."""
    keep = np.random.default_rng(seed).random(V.shape) < density
    return np.where(keep, V, 0.0)


def _check(oracle, method, V, W0, H0, iters, **kw):
    ref = oracle.nmf_method(method, V, W0, H0, iters, **kw)
    got = nmf_rs.nmf(sp.csr_matrix(V), W0.shape[1], method, W0=W0, H0=H0, max_iter=iters, **kw)
    assert got.n_iter == ref["n_iter"]
    dW, dH = rel_max(got.W, ref["W"]), rel_max(got.H, ref["H"])
    assert dW <= FACTOR_TOL, dW
    assert dH <= FACTOR_TOL, dH
    d_obj = _rel_obj(method, V, _objective(oracle, method, V, got.W, got.H),
                     _objective(oracle, method, V, ref["W"], ref["H"]))
    assert d_obj <= OBJ_TOL, d_obj
    return got, ref


def test_pbmc_subset_lee_csr(oracle):
    """lee on the 1500 x 3000 rank-8 workload (86 % non-zero) as CSR, 100 it."""
    V, W0, H0 = synthetic.make(synthetic.PBMC_SUBSET)
    _check(oracle, "lee", V, W0, H0, 100)


@pytest.mark.parametrize("method", ["brunet", "hals"])
def test_pbmc8k_shape_csr(oracle, method):
    """brunet and hals on the 2000 x 7750 rank-10 workload as CSR, 100 it."""
    V, W0, H0 = synthetic.make(synthetic.PBMC8K_SHAPE)
    if method == "hals":
        W0, H0 = nmf_rs.nndsvd_init(V, 10, fill="mean", seed=0)
    _check(oracle, method, V, W0, H0, 100)


@pytest.mark.parametrize("method", ["lee", "brunet", "hals", "dnmf"])
@pytest.mark.parametrize("density", [0.1, 0.02])
def test_sparse_matrices(oracle, method, density):
    """10 % and 2 % dense V (empty rows and columns included at 2 %)."""
    V = _sparsify(synthetic.counts_matrix(400, 900, 6, 0.3, seed=3), density, seed=4)
    if method in ("hals", "dnmf"):
        W0, H0 = nmf_rs.nndsvd_init(V, 6, fill="mean", seed=0)
    else:
        W0, H0 = nmf_rs.random_init(V, 6, seed=1)
    _check(oracle, method, V, W0, H0, 50)


@pytest.mark.parametrize("rank", [1, 3, 8, 13, 20, 27, 32])
def test_every_rank_bucket_csr(oracle, rank):
    V = _sparsify(synthetic.counts_matrix(150, 260, 6, 0.3, seed=rank), 0.3, seed=rank)
    W0, H0 = nmf_rs.random_init(V, rank, seed=rank)
    for method in ("lee", "brunet"):
        _check(oracle, method, V, W0, H0, 10)


@pytest.mark.parametrize("method", ["lee", "brunet"])
def test_stationary_deviances_csr(oracle, method):
    """The objective of every iteration (stored-entry pass + closed forms)
    against the oracle's dense objective."""
    V = _sparsify(synthetic.counts_matrix(300, 500, 5, 0.3, seed=9), 0.25, seed=2)
    W0, H0 = nmf_rs.random_init(V, 5, seed=5)
    kw = dict(stop="stationary", stationary_th=1e-4, check_interval=5, check_niter=4)
    got, ref = _check(oracle, method, V, W0, H0, 200, **kw)
    assert got.deviances.size == len(ref["deviances"]) == got.n_iter + 1
    assert max(rel(a, b) for a, b in zip(got.deviances, ref["deviances"])) <= OBJ_TOL


def test_all_zero_and_tiny(oracle):
    """An all-zero V (nnz = 0) and single-row / single-column shapes.  For
    brunet an all-zero V makes the reference's own loop divide 0 by 0 (H
    becomes 0, then rowsum(H) = 0 divides the W update), so there the NaNs
    must fall where the oracle's do."""
    for shape in ((40, 30), (1, 50), (50, 1)):
        V = np.zeros(shape)
        W0, H0 = nmf_rs.random_init(V, 2, seed=0, max_value=1.0)
        _check(oracle, "lee", V, W0, H0, 5)
        ref = oracle.nmf_method("brunet", V, W0, H0, 5)
        got = nmf_rs.nmf(sp.csr_matrix(V), 2, "brunet", W0=W0, H0=H0, max_iter=5)
        np.testing.assert_array_equal(np.isnan(got.W), np.isnan(ref["W"]))
        np.testing.assert_array_equal(np.isnan(got.H), np.isnan(ref["H"]))
        ok = ~np.isnan(ref["H"])
        np.testing.assert_allclose(got.H[ok], ref["H"][ok], rtol=0, atol=1e-300)
    V = _sparsify(synthetic.counts_matrix(1, 80, 2, 0.3, seed=1), 0.5, seed=1)
    W0, H0 = nmf_rs.random_init(V, 2, seed=0)
    _check(oracle, "lee", V, W0, H0, 5)


def test_csr_equals_dense_gpu_run():
    """The CSR and dense GPU paths agree (different summation orders only)."""
    V = _sparsify(synthetic.counts_matrix(500, 700, 5, 0.3, seed=6), 0.3, seed=6)
    W0, H0 = nmf_rs.random_init(V, 5, seed=2)
    for method in ("lee", "brunet"):
        a = nmf_rs.nmf(V, 5, method, W0=W0, H0=H0, max_iter=30)
        b = nmf_rs.nmf(sp.csr_matrix(V), 5, method, W0=W0, H0=H0, max_iter=30)
        assert rel_max(b.W, a.W) <= FACTOR_TOL
        assert rel_max(b.H, a.H) <= FACTOR_TOL


def test_csr_bit_reproducible():
    V = sp.csr_matrix(_sparsify(synthetic.counts_matrix(300, 400, 4, 0.3, seed=7), 0.2, seed=7))
    W0, H0 = nmf_rs.random_init(V.toarray(), 4, seed=3)
    a = nmf_rs.nmf(V, 4, "brunet", W0=W0, H0=H0, max_iter=40)
    b = nmf_rs.nmf(V, 4, "brunet", W0=W0, H0=H0, max_iter=40)
    np.testing.assert_array_equal(a.W, b.W)
    np.testing.assert_array_equal(a.H, b.H)


def _device_csr(V):
    import torch

    indptr, indices, data, _ = _native.csr_arrays(sp.csr_matrix(V))
    return (torch.from_numpy(indptr).cuda(), torch.from_numpy(indices).cuda(),
            torch.from_numpy(data).cuda())


def test_device_entry_matches_host_entry(oracle):
    import torch

    V = _sparsify(synthetic.counts_matrix(300, 450, 5, 0.3, seed=8), 0.15, seed=8)
    W0, H0 = nmf_rs.random_init(V, 5, seed=4)
    ref = oracle.nmf_method("brunet", V, W0, H0, 30)
    ip, ix, dv = _device_csr(V)
    dW = torch.from_numpy(W0.copy()).cuda()
    dH = torch.from_numpy(H0.copy()).cuda()
    ctx = _native.Context(0)
    o = _native.default_options()
    o.method = _native.parse_method("brunet")
    o.max_iter = 30
    nd, ni = ctypes.c_int64(0), ctypes.c_int64(0)
    _native.check(_native.load().nmfcu_run_csr_device(
        ctx.handle, ctypes.byref(o), V.shape[0], V.shape[1], 5, dv.numel(),
        ctypes.c_void_p(ip.data_ptr()), ctypes.c_void_p(ix.data_ptr()),
        ctypes.c_void_p(dv.data_ptr()), ctypes.c_void_p(dW.data_ptr()),
        ctypes.c_void_p(dH.data_ptr()), None, ctypes.byref(nd), ctypes.byref(ni),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    ctx.close()
    assert ni.value == 30
    assert rel_max(dW.cpu().numpy(), ref["W"]) <= FACTOR_TOL
    assert rel_max(dH.cpu().numpy(), ref["H"]) <= FACTOR_TOL


def test_device_entry_rejects_bad_structure():
    """A malformed device CSR is caught by the on-device check before any
    kernel indexes with it."""
    import torch

    V = _sparsify(synthetic.counts_matrix(50, 60, 3, 0.3, seed=1), 0.3, seed=1)
    ip, ix, dv = _device_csr(V)
    ctx = _native.Context(0)
    o = _native.default_options()
    o.method = _native.parse_method("lee")
    o.max_iter = 3
    dW = torch.ones((50, 3), dtype=torch.float64, device="cuda")
    dH = torch.ones((3, 60), dtype=torch.float64, device="cuda")
    nd, ni = ctypes.c_int64(0), ctypes.c_int64(0)

    def call(ip_, ix_):
        _native.check(_native.load().nmfcu_run_csr_device(
            ctx.handle, ctypes.byref(o), 50, 60, 3, dv.numel(), ctypes.c_void_p(ip_.data_ptr()),
            ctypes.c_void_p(ix_.data_ptr()), ctypes.c_void_p(dv.data_ptr()),
            ctypes.c_void_p(dW.data_ptr()), ctypes.c_void_p(dH.data_ptr()), None,
            ctypes.byref(nd), ctypes.byref(ni), None))

    bad_ix = ix.clone()
    bad_ix[3] = 60
    with pytest.raises(ValueError, match="outside"):
        call(ip, bad_ix)
    bad_ip = ip.clone()
    bad_ip[5] = bad_ip[6] + 1
    with pytest.raises(ValueError, match="non-decreasing"):
        call(bad_ip, ix)
    ctx.close()
