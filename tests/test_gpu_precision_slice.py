"""The precision forms at the atlas scale's row count: a 20000 x 20000 column
slice of the 20000 x 200000 rank-20 workload (V is 3.2 GB in f64, larger
than L2), 25 iterations from an NNDSVD start computed in f64, run on device
pointers like the benchmark.  Each mixed-precision result is compared with
the plain f64 run of the same inputs on the GPU (itself held to the oracle
at 1e-10 by the parity tests).

Bounds, written per check: relative objective <= 1e-5 (the precision
form's stated accuracy) and max|dW| / max|W| <= 1e-4."""
from __future__ import annotations

import pytest

from nmf_rs import _native, synthetic

pytestmark = pytest.mark.gpu

N, P, K, ALPHA, R, ITERS = 20000, 20000, 20, 0.2, 20, 25
REL_OBJ_TOL = 1e-5
FACTOR_TOL = 1e-4


@pytest.fixture(scope="module")
def atlas_slice():
    import torch

    from nmf_rs import nndsvd

    dev = torch.device("cuda", 0)
    V64, ld64, V32, ld32, _, _ = synthetic.device_workload(N, P, K, ALPHA, R, 99, dev)
    W0, H0 = nndsvd.nndsvd_device(V64[:, :P], R, fill="mean", seed=0)
    yield V64, ld64, V32, ld32, W0.contiguous(), H0.contiguous()
    del V64, V32
    torch.cuda.empty_cache()


def _objective(V64, W, H, method):
    import torch

    total = torch.zeros((), dtype=torch.float64, device=V64.device)
    for c0 in range(0, P, 4096):
        v = V64[:, c0:min(P, c0 + 4096)]
        wh = W @ H[:, c0:min(P, c0 + 4096)]
        if method == "brunet":
            pos = v > 0
            good = pos & (wh > 0)
            t = torch.where(good, v * torch.log(torch.where(good, v / wh, 1.0)) - v + wh,
                            torch.zeros_like(v))
            total += torch.where(pos, t, wh).sum()
        else:
            total += ((v - wh) ** 2).sum()
    return float(total) * (1.0 if method == "brunet" else 0.5)


def _run(ctx, method, precision, data):
    V64, ld64, V32, ld32, W0, H0 = data
    o = _native.default_options()
    o.method = _native.parse_method(method)
    o.precision = _native.PRECISIONS[precision]
    o.max_iter = ITERS
    W, H = W0.clone(), H0.clone()
    if precision == "fp32":
        ctx.run(o, N, P, R, V32.data_ptr(), _native.F32, ld32, W.data_ptr(), H.data_ptr(),
                v64_ptr=V64.data_ptr(), ldv64=ld64)
    else:
        ctx.run(o, N, P, R, V64.data_ptr(), _native.F64, ld64, W.data_ptr(), H.data_ptr())
    return W, H


@pytest.mark.parametrize("method,precision", [("lee", "bf16x3"), ("brunet", "bf16x3"),
                                              ("lee", "fp32")])
def test_precision_form_on_atlas_slice(atlas_slice, method, precision):
    ctx = _native.Context(0)
    try:
        W64, H64 = _run(ctx, method, "fp64", atlas_slice)
        Wm, Hm = _run(ctx, method, precision, atlas_slice)
    finally:
        ctx.close()
    V64 = atlas_slice[0]
    o64 = _objective(V64, W64, H64, method)
    om = _objective(V64, Wm, Hm, method)
    rel_obj = abs(om - o64) / abs(o64)
    rel_w = float((Wm - W64).abs().max() / W64.abs().max())
    assert rel_obj <= REL_OBJ_TOL, (rel_obj, rel_w)
    assert rel_w <= FACTOR_TOL, (rel_obj, rel_w)
