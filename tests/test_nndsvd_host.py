"""The NNDSVD start's host logic (randomized range finder, LU / QR / SVD
normalisations, sign fixing, the non-negative split and the fills) against
fixtures made by the reference's own ``nndsvd_init`` (tests/golden/
make_nndsvd_golden.py).  The passes over V are plain torch products on the
CPU here; the GPU tests run the same logic on the CUDA library's passes.

Tolerance: max|dW| / max|W| <= 1e-9 (and for H).  The randomized SVD is
deterministic given its test vectors; what differs is the rounding of the
products, which the power iterations and the small factorizations carry
with an amplification set by the singular value gaps of each case.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, rel_max

torch = pytest.importorskip("torch")

from nmf_rs import nndsvd  # noqa: E402

CASES = ["quickstart_mean", "quickstart_zero", "wide_eps", "tiny_mean", "rank30_mean"]
TOL = 1e-9


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


def _cpu_product(V):
    Vt = torch.from_numpy(np.ascontiguousarray(V))

    def product(trans, X):
        return Vt.T @ X if trans else Vt @ X

    return product


@pytest.mark.parametrize("name", CASES)
def test_host_logic_matches_reference_nndsvd(golden, name):
    V, rank, fill, seed, over, W_ref, H_ref = golden[name]
    Vt = torch.from_numpy(V)
    W, H = nndsvd.nndsvd_device(Vt, rank, fill=fill, seed=seed, n_oversamples=over,
                                product=_cpu_product(V))
    assert W.shape == W_ref.shape and H.shape == H_ref.shape
    assert rel_max(W.numpy(), W_ref) <= TOL, rel_max(W.numpy(), W_ref)
    assert rel_max(H.numpy(), H_ref) <= TOL, rel_max(H.numpy(), H_ref)


def test_lu_pl_reproduces_the_matrix():
    gen = np.random.default_rng(0)
    for shape in [(50, 7), (7, 12), (1, 3), (9, 9)]:
        X = torch.from_numpy(gen.normal(size=shape))
        PL = nndsvd._lu_pl(X)
        LU, piv, _ = torch.linalg.lu_factor_ex(X)
        U = torch.triu(LU[: min(shape), :])
        np.testing.assert_allclose((PL @ U).numpy(), X.numpy(), rtol=0, atol=1e-13)


def test_fill_validation():
    with pytest.raises(ValueError, match="fill"):
        nndsvd.nndsvd_device(torch.ones((4, 5), dtype=torch.float64), 2, fill="bogus",
                             product=_cpu_product(np.ones((4, 5))))
