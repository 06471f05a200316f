"""Fixed-length runs replay their main iterations as a CUDA graph when the
stream can be captured (the library's own stream behind nmf(), a side
stream on the device entry) and the per-kernel timing is off.  The graph
holds the same kernels in the same order as launching every iteration, so
the results must be the same bits; on the default stream (not capturable)
every iteration is launched directly."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_max

import nmf_rs
from nmf_rs import _native, synthetic

pytestmark = pytest.mark.gpu


def _device_run(method, V, W0, H0, iters, precision, stream):
    n, p = V.shape
    r = W0.shape[1]
    dev = torch.device("cuda", 0)
    Vd = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
    Wd = torch.from_numpy(np.ascontiguousarray(W0)).to(dev)
    Hd = torch.from_numpy(np.ascontiguousarray(H0)).to(dev)
    o = _native.default_options()
    o.method = _native.parse_method(method)
    o.stop = 0
    o.max_iter = iters
    o.precision = _native.PRECISIONS[precision]
    o.device = 0
    ctx = _native.Context(0)
    try:
        ctx.run(o, n, p, r, Vd.data_ptr(), _native.F64, p, Wd.data_ptr(), Hd.data_ptr(),
                stream=stream.cuda_stream if stream is not None else 0)
        torch.cuda.synchronize()
        return Wd.cpu().numpy(), Hd.cpu().numpy(), ctx.launch_count()
    finally:
        ctx.close()


@pytest.mark.parametrize("method,precision", [("brunet", "fp64"), ("lee", "fp64"),
                                              ("hals", "fp64"), ("brunet", "bf16x3"),
                                              ("lee", "bf16x3")])
def test_graph_replay_equals_direct_launches(oracle, method, precision):
    V = synthetic.counts_matrix(300, 700, 5, 0.3, seed=12)
    W0, H0 = nmf_rs.random_init(V, 6, seed=4)
    iters = 57  # iteration 1, five replays of ten, six more; brunet clamps inside
    side = torch.cuda.Stream(torch.device("cuda", 0))
    Wg, Hg, lg = _device_run(method, V, W0, H0, iters, precision, side)
    Wd, Hd, ld = _device_run(method, V, W0, H0, iters, precision, None)
    np.testing.assert_array_equal(Wg, Wd)
    np.testing.assert_array_equal(Hg, Hd)
    assert lg == ld  # the graph's launches are counted like direct ones
    if precision == "fp64" and method != "hals":
        ref = oracle.nmf_method(method, V, W0, H0, iters)
        assert rel_max(Wg, ref["W"]) <= 1e-10
        assert rel_max(Hg, ref["H"]) <= 1e-10


def test_host_entry_uses_the_graph_and_matches_the_oracle(oracle):
    # nmf() runs on the library's own stream (capturable).
    V = synthetic.counts_matrix(250, 400, 4, 0.3, seed=2)
    W0, H0 = nmf_rs.random_init(V, 5, seed=8)
    got = nmf_rs.nmf(V, 5, "brunet", W0=W0, H0=H0, max_iter=80)
    ref = oracle.nmf_method("brunet", V, W0, H0, 80)
    assert rel_max(got.W, ref["W"]) <= 1e-10
    assert rel_max(got.H, ref["H"]) <= 1e-10
