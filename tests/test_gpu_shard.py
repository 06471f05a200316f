"""Column shards on the CUDA library (nmfcu_shard_*), on one GPU.

Several shards of one V run in one process, in lockstep on one stream; the
all-reduce between the halves of an iteration is an explicit sum of the
shards' device buffers (no kernel waits on another shard).  This exercises
every device-side step of the multi-GPU path; the collective itself is
covered by the gloo tests on CPU.

Tolerances: FP64 factors max|d| / max|ref| <= 1e-10 against the oracle;
reduced precisions: objective within 1e-5 (relative) of the FP64 oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rel, rel_max

import nmf_rs
from nmf_rs import _native, nndsvd, shard, synthetic

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _opts(method, max_iter, precision="fp64", **kw):
    o = _native.default_options()
    o.method = _native.parse_method(method)
    o.max_iter = max_iter
    o.precision = _native.PRECISIONS[precision]
    if method == "dnmf":
        o.sparsity_h = o.sparsity_w = 0.01
    if kw.get("stop") == "stationary":
        o.stop = 1
        o.stationary_th = kw["stationary_th"]
        o.check_interval = kw["check_interval"]
        o.check_niter = kw["check_niter"]
    return o


def run_local(V, W0, H0, method, parts, max_iter, precision="fp64", **kw):
    """`parts` shards of V on one GPU in lockstep; returns W, H, n_iter, dev."""
    Vd = nndsvd.upload(V)
    p = V.shape[1]
    o = _opts(method, max_iter, precision, **kw)
    blocks = [shard.split_columns(p, parts, q) for q in range(parts)]
    shards = [shard.DeviceShard(Vd[:, c0:c1], W0, H0[:, c0:c1], o) for c0, c1 in blocks]

    def reduce(attr):
        total = getattr(shards[0], attr).clone()
        for sh in shards[1:]:
            total += getattr(sh, attr)
        for sh in shards:
            getattr(sh, attr).copy_(total)

    class Lockstep:
        """All shards as one object with the shard step interface."""
        reduce_buffer = "reduce_buffer"
        objective = "objective"

        def step(self, phase):
            for sh in shards:
                sh.step(phase)

        def status(self):
            st = [sh.status() for sh in shards]
            assert len(set(st)) == 1  # every shard took the same stop decision
            return st[0]

    n_iter, _ = shard.run_shard(Lockstep(), reduce, max_iter, o.stop == 1)
    results = [sh.result() for sh in shards]
    W = results[0][0].cpu().numpy()
    for r_ in results[1:]:
        np.testing.assert_array_equal(r_[0].cpu().numpy(), W)  # identical copies of W
    H = np.concatenate([r_[1].cpu().numpy() for r_ in results], axis=1)
    dev = results[0][2].cpu().numpy()
    for sh in shards:
        sh.close()
    return W, H, n_iter, dev


@pytest.mark.parametrize("method", ["lee", "brunet", "hals", "dnmf"])
@pytest.mark.parametrize("parts", [1, 2, 3])
def test_shards_match_the_oracle(oracle, method, parts):
    V = synthetic.counts_matrix(300, 700, 6, 0.3, seed=5)
    W0, H0 = nmf_rs.random_init(V, 7, seed=2)
    if method in ("hals", "dnmf"):  # a well-conditioned start (HALS amplifies rounding)
        W0, H0 = nmf_rs.nndsvd_init(V, 7, fill="mean", seed=0)
    W, H, n_iter, _ = run_local(V, W0, H0, method, parts, 30)
    ref = oracle.nmf_method(method, V, W0, H0, 30)
    assert n_iter == 30
    assert rel_max(W, ref["W"]) <= TOL, rel_max(W, ref["W"])
    assert rel_max(H, ref["H"]) <= TOL, rel_max(H, ref["H"])


def test_one_shard_equals_the_single_solve(quickstart):
    V, W0, H0 = quickstart
    W, H, _, _ = run_local(V, W0, H0, "lee", 1, 50)
    got = nmf_rs.nmf(V, 5, "lee", W0=W0, H0=H0, max_iter=50)
    assert rel_max(W, got.W) <= 1e-14 and rel_max(H, got.H) <= 1e-14


@pytest.mark.parametrize("method", ["lee", "brunet"])
def test_shards_stationary(oracle, quickstart, method):
    V, W0, H0 = quickstart
    kw = dict(stop="stationary", stationary_th=1.0, check_interval=10, check_niter=3)
    W, H, n_iter, dev = run_local(V, W0, H0, method, 3, 400, **kw)
    ref = oracle.nmf_method(method, V, W0, H0, 400, **kw)
    assert n_iter == ref["n_iter"] < 400
    assert dev.size == ref["deviances"].size
    assert np.max(np.abs(dev - ref["deviances"]) / np.abs(ref["deviances"])) <= TOL
    assert rel_max(W, ref["W"]) <= TOL


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
@pytest.mark.parametrize("method", ["lee", "brunet"])
def test_shards_reduced_precision(oracle, method, precision):
    V, W0, H0 = synthetic.make(synthetic.PBMC_SUBSET)
    W, H, _, _ = run_local(V, W0, H0, method, 2, 40, precision)
    ref = oracle.nmf_method(method, V, W0, H0, 40)
    obj = oracle.kl_divergence if method == "brunet" else oracle.euclidean_distance
    assert rel(obj(V, W, H), obj(V, ref["W"], ref["H"])) <= 1e-5


def test_nmf_sharded_single_process(quickstart):
    V, W0, H0 = quickstart
    W, H, n_iter, _ = shard.nmf_sharded(nndsvd.upload(V), 5, "lee", W0=W0, H0_local=H0,
                                        max_iter=20)
    got = nmf_rs.nmf(V, 5, "lee", W0=W0, H0=H0, max_iter=20)
    assert n_iter == 20
    assert rel_max(W.cpu().numpy(), got.W) <= 1e-14
    assert rel_max(H.cpu().numpy(), got.H) <= 1e-14


def test_shard_rejects_other_methods(quickstart):
    V, W0, H0 = quickstart
    with pytest.raises(NotImplementedError):
        shard.nmf_sharded(nndsvd.upload(V), 5, "offset", W0=W0, H0_local=H0, max_iter=2)


@pytest.mark.parametrize("method", ["lee", "brunet"])
def test_shards_with_empty_blocks(oracle, method):
    # p = 40 over 5 shards: blocks of 0, 16, 0, 16 and 8 columns
    V = synthetic.counts_matrix(90, 40, 4, 0.3, seed=12) + 0.01
    W0, H0 = nmf_rs.random_init(V, 5, seed=1)
    W, H, n_iter, _ = run_local(V, W0, H0, method, 5, 15)
    ref = oracle.nmf_method(method, V, W0, H0, 15)
    assert rel_max(W, ref["W"]) <= TOL and rel_max(H, ref["H"]) <= TOL
