"""Column-sharded solve (nmf_rs.shard.run_shard) over 2 gloo ranks on CPU,
with the numpy step engine, against the single-process oracle.

Checks: the column split, that every rank takes the same collective steps
and stops at the same iteration, identical W on every rank, and parity of
W, the gathered H and the deviances with the oracle (max|d| / max|ref| <=
1e-10: the sums over columns are grouped per rank).
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import GOLDEN, rel_max

from nmf_rs import shard

TOL = 1e-10


def test_split_columns_covers_and_aligns():
    for p in (1, 15, 16, 17, 60, 1000, 200000):
        for world in (1, 2, 3, 8):
            blocks = [shard.split_columns(p, world, q) for q in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == p
            for (a0, a1), (b0, b1) in zip(blocks, blocks[1:]):
                assert a1 == b0
            for c0, c1 in blocks:
                assert c0 % shard.ALIGN == 0 and c0 <= c1
    with pytest.raises(ValueError):
        shard.split_columns(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, method, kw, out_dir):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [here]
    from shard_numpy_engine import NumpyShard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        z = np.load(os.path.join(out_dir, "inputs.npz"))
        V, W0, H0 = z["V"], z["W0"], z["H0"]
        c0, c1 = shard.split_columns(V.shape[1], world, rank)
        eng = NumpyShard(V[:, c0:c1], W0, H0[:, c0:c1], method, **kw)
        n_iter, stopped = shard.run_shard(eng, shard.torch_reduce(), kw["max_iter"],
                                          kw.get("stop") == "stationary")
        W, H, dev = eng.result()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), W=W, H=H, dev=dev, n_iter=n_iter,
                 c0=c0, c1=c1)
    finally:
        dist.destroy_process_group()


def _run(tmp_path, method, V, W0, H0, world=2, **kw):
    np.savez(tmp_path / "inputs.npz", V=V, W0=W0, H0=H0)
    mp.start_processes(_worker, args=(world, _free_port(), method, kw, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    parts = [np.load(tmp_path / f"rank{q}.npz") for q in range(world)]
    H = np.zeros_like(H0)
    for z in parts:
        H[:, int(z["c0"]):int(z["c1"])] = z["H"]
    for z in parts[1:]:
        np.testing.assert_array_equal(parts[0]["W"], z["W"])  # identical copies of W
        assert int(parts[0]["n_iter"]) == int(z["n_iter"])
    return parts[0]["W"], H, int(parts[0]["n_iter"]), parts[0]["dev"]


@pytest.fixture(scope="module")
def start(oracle):
    z = np.load(GOLDEN / "quickstart_inputs.npz")
    V, W0, H0 = z["V"], z["W0"], z["H0"]
    # HALS from a random start is ill conditioned; 30 lee iterations first.
    warm = oracle.nmf_method("lee", V, W0, H0, 30)
    return V, W0, H0, warm["W"], warm["H"]


@pytest.mark.parametrize("method", ["lee", "brunet", "hals", "dnmf"])
def test_two_gloo_ranks_match_the_oracle(tmp_path, oracle, start, method):
    V, W0, H0, Wl, Hl = start
    if method in ("hals", "dnmf"):
        W0, H0 = Wl, Hl
    kw = dict(max_iter=25)
    W, H, n_iter, _ = _run(tmp_path, method, V, W0, H0, **kw)
    ref = oracle.nmf_method(method, V, W0, H0, 25)
    assert n_iter == 25
    assert rel_max(W, ref["W"]) <= TOL, rel_max(W, ref["W"])
    assert rel_max(H, ref["H"]) <= TOL, rel_max(H, ref["H"])


@pytest.mark.parametrize("method", ["lee", "brunet"])
def test_two_gloo_ranks_stationary_stop(tmp_path, oracle, start, method):
    V, W0, H0, _, _ = start
    kw = dict(max_iter=400, stop="stationary", stationary_th=1.0, check_interval=10,
              check_niter=3)
    W, H, n_iter, dev = _run(tmp_path, method, V, W0, H0, **kw)
    ref = oracle.nmf_method(method, V, W0, H0, 400, **{k: v for k, v in kw.items()
                                                        if k != "max_iter"})
    assert n_iter == ref["n_iter"] < 400
    assert dev.size == ref["deviances"].size
    assert np.max(np.abs(dev - ref["deviances"]) / np.abs(ref["deviances"])) <= TOL
    assert rel_max(W, ref["W"]) <= TOL


@pytest.mark.parametrize("method", ["lee", "brunet"])
def test_three_gloo_ranks_uneven_blocks(tmp_path, oracle, start, method):
    V, W0, H0, _, _ = start  # 60 columns: blocks of 16, 16 and 28
    W, H, n_iter, _ = _run(tmp_path, method, V, W0, H0, world=3, max_iter=15)
    ref = oracle.nmf_method(method, V, W0, H0, 15)
    assert n_iter == 15
    assert rel_max(W, ref["W"]) <= TOL and rel_max(H, ref["H"]) <= TOL


def test_gloo_rank_with_no_columns(tmp_path, oracle, start):
    # 20 columns over 3 ranks: rank 0 holds none, yet takes every collective step
    V, W0, H0, _, _ = start
    V, H0 = V[:, :20].copy(), H0[:, :20].copy()
    W, H, n_iter, _ = _run(tmp_path, "lee", V, W0, H0, world=3, max_iter=10)
    ref = oracle.nmf_method("lee", V, W0, H0, 10)
    assert rel_max(W, ref["W"]) <= TOL and rel_max(H, ref["H"]) <= TOL
