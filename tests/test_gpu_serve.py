"""The serving form on the GPU: each request's result is the one nmf()
gives for the same arguments alone -- bit for bit, since a request runs the
single-solve engine on its own stream with a plan that depends only on its
shape -- whatever else is in flight; admission keeps the slots' device
memory within the budget; cancellation and per-request errors."""
from __future__ import annotations

import concurrent.futures
import threading

import numpy as np
import pytest

import nmf_rs
from nmf_rs import serve, synthetic

pytestmark = pytest.mark.gpu

# (n, p, rank, method, precision, iters, stop)
MIX = [
    (120, 300, 3, "brunet", "fp64", 40, "max_iter"),
    (257, 513, 7, "lee", "fp64", 60, "max_iter"),
    (600, 1100, 12, "hals", "fp64", 30, "max_iter"),
    (300, 2000, 5, "dnmf", "fp64", 25, "max_iter"),
    (1000, 2500, 20, "brunet", "fp32", 50, "max_iter"),
    (800, 1500, 10, "lee", "fp32", 45, "max_iter"),
    (150, 4000, 4, "brunet", "fp64", 120, "stationary"),
    (2000, 700, 16, "lee", "fp64", 35, "max_iter"),
    (64, 64, 2, "hals", "fp64", 80, "max_iter"),
    (1500, 3000, 8, "lee", "fp64", 100, "max_iter"),
    (400, 900, 30, "brunet", "fp64", 20, "max_iter"),
    (333, 777, 9, "dnmf", "fp32", 40, "max_iter"),
]


def _case(i, n, p, rank, seed_off=0):
    V = synthetic.counts_matrix(n, p, max(2, rank // 2), 0.3, 100 + i + seed_off)
    W0, H0 = nmf_rs.random_init(V, rank, seed=7 + i)
    return V, W0, H0


def _kw(method, precision, iters, stop):
    kw = dict(max_iter=iters, precision=precision, stop=stop)
    if stop == "stationary":
        kw.update(check_interval=10, check_niter=3, stationary_th=1e-9)
    return kw


@pytest.fixture(scope="module")
def mix():
    cases = []
    for i, (n, p, r, m, prec, it, stop) in enumerate(MIX):
        V, W0, H0 = _case(i, n, p, r)
        alone = nmf_rs.nmf(V, r, m, W0=W0, H0=H0, **_kw(m, prec, it, stop))
        cases.append((V, W0, H0, r, m, _kw(m, prec, it, stop), alone))
    return cases


def _same(res, alone):
    assert res.n_iter == alone.n_iter
    np.testing.assert_array_equal(res.W, alone.W)
    np.testing.assert_array_equal(res.H, alone.H)
    np.testing.assert_array_equal(res.deviances, alone.deviances)


def test_each_result_in_the_mix_equals_alone(mix):
    with serve.Server(slots=4) as srv:
        reqs = [srv.submit(V, r, m, W0=W0, H0=H0, **kw) for V, W0, H0, r, m, kw, _ in mix]
        for req, case in zip(reqs, mix):
            _same(req.result(timeout=120), case[-1])
        st = srv.stats()
    assert st["completed"] == len(mix) and st["failed"] == 0
    assert st["peak_running"] >= 2  # requests overlapped on the device
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["iterations"] == sum(c[-1].n_iter for c in mix)
    assert st["peak_bytes"] <= st["budget_bytes"]


def test_submissions_from_many_threads(mix):
    with serve.Server(slots=3) as srv:
        def one(case):
            V, W0, H0, r, m, kw, alone = case
            _same(srv.submit(V, r, m, W0=W0, H0=H0, **kw).result(timeout=120), alone)
        with concurrent.futures.ThreadPoolExecutor(6) as ex:
            list(ex.map(one, mix * 2))
        assert srv.stats()["completed"] == 2 * len(mix)


def test_admission_keeps_memory_within_the_budget():
    V, W0, H0 = _case(0, 1500, 3000, 10)
    alone = nmf_rs.nmf(V, 10, "lee", W0=W0, H0=H0, max_iter=30)
    with serve.Server(slots=1) as srv:  # footprint of one such request
        srv.submit(V, 10, "lee", W0=W0, H0=H0, max_iter=30).result(timeout=120)
        footprint = srv.stats()["in_use_bytes"]
    assert footprint > 8 * V.size  # V's device copy at least
    budget = int(1.5 * footprint)  # room for one request at a time
    with serve.Server(slots=3, budget_bytes=budget) as srv:
        reqs = [srv.submit(V, 10, "lee", W0=W0, H0=H0, max_iter=30) for _ in range(4)]
        for q in reqs:
            _same(q.result(timeout=120), alone)
        st = srv.stats()
    assert st["peak_running"] == 1
    assert st["peak_bytes"] <= budget


def test_request_larger_than_the_budget_is_refused():
    V, W0, H0 = _case(1, 500, 800, 5)
    with serve.Server(slots=2, budget_bytes=1 << 20) as srv:
        with pytest.raises(MemoryError):
            srv.submit(V, 5, "lee", W0=W0, H0=H0, max_iter=5)


def test_cancel_a_queued_request():
    V, W0, H0 = _case(2, 2000, 6000, 16)
    small = _case(3, 100, 200, 3)
    with serve.Server(slots=1) as srv:
        first = srv.submit(V, 16, "brunet", W0=W0, H0=H0, max_iter=300)
        queued = srv.submit(small[0], 3, "lee", W0=small[1], H0=small[2], max_iter=10)
        assert queued.cancel()
        with pytest.raises(concurrent.futures.CancelledError):
            queued.result(timeout=60)
        assert first.result(timeout=300).n_iter == 300
        st = srv.stats()
    assert st["cancelled"] == 1 and st["completed"] == 1


def test_argument_errors_are_raised_at_submit():
    V, W0, H0 = _case(4, 50, 60, 3)
    with serve.Server(slots=1) as srv:
        with pytest.raises(ValueError):
            srv.submit(V, 3, "nope", W0=W0, H0=H0, max_iter=5)
        with pytest.raises(ValueError):
            srv.submit(-V - 1, 3, "lee", W0=W0, H0=H0, max_iter=5)
        ok = srv.submit(V, 3, "lee", W0=W0, H0=H0, max_iter=5).result(timeout=60)
    assert ok.n_iter == 5


def test_wait_with_a_short_timeout_keeps_the_request():
    V, W0, H0 = _case(5, 2000, 8000, 20)
    with serve.Server(slots=1) as srv:
        q = srv.submit(V, 20, "brunet", W0=W0, H0=H0, max_iter=200)
        try:
            q.result(timeout=0)
        except TimeoutError:
            pass  # still running: the request stays valid
        assert q.result(timeout=300).n_iter == 200
