"""GPU NNDSVD start: the V contraction of the CUDA library
(``nmfcu_v_product_device``) against torch f64 products, and ``nndsvd_init``
against fixtures made by the reference's own ``nndsvd_init``
(tests/golden/make_nndsvd_golden.py).

Tolerances: products max|d| / max|ref| <= 1e-12 (FP64, sums in another
order); NNDSVD factors max|d| / max|ref| <= 1e-9 (the products' rounding
carried through the power iterations; the CPU run of the same host logic
agrees with the fixtures to 2e-13).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, rel_max

import nmf_rs
from nmf_rs import _native, nndsvd, synthetic

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

PROD_TOL = 1e-12
NNDSVD_TOL = 1e-9
CASES = ["quickstart_mean", "quickstart_zero", "wide_eps", "tiny_mean", "rank30_mean"]


def _product(V, X, trans, ldv=None):
    """V (host n x p) with row pitch ldv on the device, X (host) -> device product."""
    n, p = V.shape
    ldv = ldv or p
    buf = torch.zeros((n, max(ldv, 1)), dtype=torch.float64, device="cuda")
    buf[:, :p] = torch.from_numpy(V)
    Xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    l = X.shape[1]
    out = torch.full((p if trans else n, l), np.nan, dtype=torch.float64, device="cuda")
    ctx = nndsvd._context(0)
    ctx.v_product(trans, n, p, l, buf.data_ptr(), ldv, Xd.data_ptr(), l, out.data_ptr(), l,
                  torch.cuda.current_stream().cuda_stream)
    return out.cpu().numpy()


@pytest.mark.parametrize("shape", [(1000, 777, 17), (300, 2049, 40), (1, 50, 3), (64, 1, 5),
                                   (513, 129, 1), (257, 1031, 64)])
@pytest.mark.parametrize("trans", [0, 1])
def test_v_product_matches_torch(shape, trans):
    n, p, l = shape
    gen = np.random.default_rng(n * 7 + p + l)
    V = synthetic.counts_matrix(n, p, 4, 0.3, seed=n + p)
    X = gen.normal(size=(n if trans else p, l))
    got = _product(V, X, trans)
    ref = V.T @ X if trans else V @ X
    assert rel_max(got, ref) <= PROD_TOL, rel_max(got, ref)


def test_v_product_pitched_and_unaligned():
    V = synthetic.counts_matrix(200, 301, 4, 0.3, seed=1)
    X = np.random.default_rng(0).normal(size=(301, 9))
    ref = V @ X
    assert rel_max(_product(V, X, 0, ldv=320), ref) <= PROD_TOL  # padded, aligned pitch
    assert rel_max(_product(V, X, 0, ldv=303), ref) <= PROD_TOL  # odd pitch: copied first


def test_v_product_argument_errors():
    ctx = nndsvd._context(0)
    with pytest.raises(ValueError):
        ctx.v_product(2, 4, 4, 1, 1, 4, 1, 1, 1, 1)
    with pytest.raises(ValueError):
        ctx.v_product(0, 4, 4, 1, 1, 3, 1, 1, 1, 1)  # ldv < p


@pytest.fixture(scope="module")
def golden(quickstart):
    z = np.load(GOLDEN / "nndsvd_cases.npz")
    out = {}
    for name in CASES:
        V = quickstart[0] if name.startswith("quickstart") else z[f"{name}__V"]
        rank, seed, over = (int(x) for x in z[f"{name}__meta"])
        out[name] = (V, rank, str(z[f"{name}__fill"]), seed, over, z[f"{name}__W"],
                     z[f"{name}__H"])
    return out


@pytest.mark.parametrize("name", CASES)
def test_nndsvd_matches_reference(golden, name):
    V, rank, fill, seed, over, W_ref, H_ref = golden[name]
    W, H = nmf_rs.nndsvd_init(V, rank, fill=fill, seed=seed, n_oversamples=over)
    assert rel_max(W, W_ref) <= NNDSVD_TOL, rel_max(W, W_ref)
    assert rel_max(H, H_ref) <= NNDSVD_TOL, rel_max(H, H_ref)


def test_nndsvd_large_against_cpu_products():
    # 3000 x 5000, rank 20: the device passes against the same host logic on
    # CPU torch products.  No all-zero row (there the factors' entries are
    # rounding noise whose sign picks between the fill and ~1e-16).
    V = synthetic.counts_matrix(3000, 5000, 30, 0.3, seed=21) + 0.01
    Vt = torch.from_numpy(V)
    W_ref, H_ref = nndsvd.nndsvd_device(
        Vt, 20, fill="mean", seed=0,
        product=lambda t, X: Vt.T @ X.cpu() if t else Vt @ X.cpu())
    W, H = nmf_rs.nndsvd_init(V, 20, fill="mean", seed=0)
    assert rel_max(W, W_ref.numpy()) <= NNDSVD_TOL
    assert rel_max(H, H_ref.numpy()) <= NNDSVD_TOL


def test_nndsvd_shapes_positive_and_repeatable(quickstart):
    V, _, _ = quickstart
    W, H = nmf_rs.nndsvd_init(V, 5, fill="mean", seed=0)
    assert W.shape == (200, 5) and H.shape == (5, 60)
    assert (W > 0).all() and (H > 0).all()
    W2, H2 = nmf_rs.nndsvd_init(V, 5, fill="mean", seed=0)
    np.testing.assert_array_equal(W, W2)
    np.testing.assert_array_equal(H, H2)


def test_nndsvd_zero_rows_get_the_fill_or_noise():
    V = synthetic.counts_matrix(80, 120, 4, 0.3, seed=3)
    V[5] = 0.0
    W, H = nmf_rs.nndsvd_init(V, 6, fill="mean", seed=0)
    m = V.mean()
    row = W[5]
    assert np.all((np.abs(row) <= 1e-12 * np.abs(W).max()) | (row == m))
    assert np.all(W >= 0) and np.all(H >= 0)


def test_nndsvd_device_resident_and_launches():
    V = synthetic.counts_matrix(500, 700, 5, 0.3, seed=4)
    Vd = nndsvd.upload(V)
    ctx = nndsvd._context(0)
    before = ctx.launch_count()
    W, H = nndsvd.nndsvd_device(Vd, 6, fill="mean", seed=0)
    assert W.is_cuda and H.is_cuda and W.shape == (500, 6) and H.shape == (6, 700)
    assert ctx.launch_count() > before  # the passes ran in the CUDA library
    assert _native.device_count() >= 1
