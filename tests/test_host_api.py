"""Host-side logic of the drop-in boundary, CPU only: the C-ABI library loads
and exports every symbol include/nmfcu.h declares, name parsing follows
Algo/Stop::from_str, the Python API validates like the reference's nmf(),
and without a GPU every compute call fails loudly (no CPU fallback)."""
from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT

import nmf_rs
from nmf_rs import _native


def _declared_symbols() -> list[str]:
    text = (ROOT / "include" / "nmfcu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nmfcu_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    declared = _declared_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), f"libnmfcu.so does not export {name}"
    # ... and the binding declares a signature for each of them.
    assert set(declared) == set(_native.SIGNATURES)


def test_abi_version():
    assert _native.load().nmfcu_abi_version() == 1


# Algo::from_str, lib.rs:1486-1505 -- every accepted spelling.
ALGO_NAMES = {
    0: ["brunet", "KL", "Brunet"],
    1: ["lee", "frobenius", "EUCLIDEAN"],
    2: ["offset"],
    3: ["nsNMF", "ns", "ns_nmf"],
    4: ["hals", "HALS"],
    5: ["ehals", "e-hals", "extrap_hals"],
    6: ["dnmf", "diag_nmf", "diagonalised_nmf", "rcppml"],
    7: ["ls-nmf", "lsNMF"],
    8: ["snmf/r", "snmf_r", "snmfr"],
    9: ["snmf/l", "snmf_l", "SNMFL"],
}


@pytest.mark.parametrize("mid,names", sorted(ALGO_NAMES.items()))
def test_parse_method(mid, names):
    for name in names:
        assert _native.parse_method(name) == mid


def test_parse_method_unknown():
    with pytest.raises(ValueError, match="unknown algorithm 'nope'"):
        _native.parse_method("nope")


def test_parse_stop():
    for name in ("max_iter", "fixed", "NONE"):
        assert _native.parse_stop(name) == 0
    assert _native.parse_stop("Stationary") == 1
    with pytest.raises(ValueError, match="unknown stopping criterion"):
        _native.parse_stop("converged")


def test_options_default_matches_reference_defaults():
    o = _native.default_options()
    assert o.eps == 1e-9 and o.rescale == 1 and o.theta == 0.5
    assert o.stationary_th == np.finfo(np.float64).eps
    assert o.check_interval == 50 and o.check_niter == 10
    assert o.sparsity_h == o.sparsity_w == o.smoothness_h == o.smoothness_w == 0.0


def test_smoothing_matrix():
    # lib.rs:2194-2206 (smoothing_diagonal).
    S = nmf_rs.smoothing_matrix(3, 0.5)
    off = 0.5 / 3.0
    expected = np.full((3, 3), off)
    np.fill_diagonal(expected, 0.5 + off)
    assert np.abs(S - expected).max() < 1e-15


def test_set_num_threads_reports_no_pool():
    assert nmf_rs.set_num_threads(4) is False


def test_random_init_stream_order():
    V = np.arange(12.0).reshape(3, 4)
    W0, H0 = nmf_rs.random_init(V, 2, seed=7)
    gen = np.random.default_rng(7)
    np.testing.assert_array_equal(W0, gen.uniform(0, 11.0, (3, 2)))
    np.testing.assert_array_equal(H0, gen.uniform(0, 11.0, (2, 4)))


def test_nndsvd_init_argument_errors_come_first(quickstart):
    # The argument checks run before the device is touched (no GPU here).
    V, _, _ = quickstart
    with pytest.raises(ValueError):
        nmf_rs.nndsvd_init(-V, 2)
    with pytest.raises(ValueError):
        nmf_rs.nndsvd_init(V, 2, fill="bogus")


# nmf() validation (python/nmf_rs/__init__.py:487-526) happens before any
# device work, so it is checked here without a GPU.
def test_nmf_validation_errors():
    V = np.ones((6, 5))
    with pytest.raises(ValueError, match="unknown method"):
        nmf_rs.nmf(V, 2, method="nope")
    with pytest.raises(ValueError, match="non-negative"):
        nmf_rs.nmf(-V, 2)
    with pytest.raises(ValueError, match="W0.shape"):
        nmf_rs.nmf(V, 2, W0=np.ones((6, 3)), H0=np.ones((2, 5)))
    with pytest.raises(ValueError, match="H0.shape"):
        nmf_rs.nmf(V, 2, W0=np.ones((6, 2)), H0=np.ones((2, 4)))
    with pytest.raises(ValueError, match="offset.shape"):
        nmf_rs.nmf(V, 2, offset=np.ones(5))
    with pytest.raises(ValueError, match="weight.shape"):
        nmf_rs.nmf(V, 2, weight=np.ones((5, 5)))
    with pytest.raises(ValueError, match="2-D"):
        nmf_rs.nmf(np.ones(5), 2)
    with pytest.raises(ValueError, match="requires a `weight`"):
        nmf_rs.nmf(V, 2, method="lsnmf")
    with pytest.raises(ValueError, match="unknown stopping"):
        nmf_rs.nmf(V, 2, stop="never")
    with pytest.raises(ValueError, match="precision"):
        nmf_rs.nmf(V, 2, precision="fp16")


def test_cv_rank_rejects_negative_v_before_any_device_work():
    with pytest.raises(ValueError, match="non-negative"):
        nmf_rs.cv_rank(-np.ones((4, 4)), [2])


def test_regularisation_routing():
    # python/nmf_rs/__init__.py:528-538
    assert nmf_rs._regularisation("dnmf", 0.3, 2.0) == (0.3, 0.3, 0.0, 0.0)
    assert nmf_rs._regularisation("snmf/r", 0.3, 2.0) == (0.3, 0.0, 0.0, 2.0)
    assert nmf_rs._regularisation("snmf/l", 0.3, 2.0) == (0.0, 0.3, 2.0, 0.0)
    assert nmf_rs._regularisation("lee", 0.3, 2.0) == (0.0, 0.0, 0.0, 0.0)


@pytest.mark.skipif(_native.available() and _native.device_count() > 0,
                    reason="a GPU is present; the no-device path is not reachable")
def test_no_gpu_fails_loudly(quickstart):
    V, W0, H0 = quickstart
    with pytest.raises(RuntimeError, match="no CUDA device"):
        nmf_rs.nmf(V, 5, W0=W0, H0=H0, max_iter=2)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        nmf_rs.update_h_lee(V, W0, H0)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        _native.Context(0)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_native, "_lib", None)
    monkeypatch.setattr(_native, "LIB_PATH", tmp_path / "libnmfcu.so")
    with pytest.raises(RuntimeError, match="CUDA backend not available"):
        nmf_rs.nmf(np.ones((4, 3)), 2, max_iter=1)


def test_synthetic_generator():
    from nmf_rs import synthetic

    V = synthetic.counts_matrix(300, 400, 6, 0.3, seed=3)
    assert V.shape == (300, 400) and V.flags.c_contiguous
    assert (V >= 0).all() and np.isfinite(V).all()
    assert 0.05 < float((V == 0).mean()) < 0.95
    np.testing.assert_array_equal(V, synthetic.counts_matrix(300, 400, 6, 0.3, seed=3))


# ---------------------------------------------------------------------------
# Batched solves and consensus: argument checks and the metrics (no GPU).
# ---------------------------------------------------------------------------

def test_batch_rejects_unsupported_before_touching_a_device():
    from nmf_rs import consensus

    V = np.ones((4, 5))
    starts = [(np.ones((4, 2)), np.ones((2, 5)))]
    with pytest.raises(NotImplementedError):
        consensus.run_batch(V, starts, 3, method="lee")
    # Ranks above the largest supported one (NMFCU_MAX_WIDE_RANK, 256).
    with pytest.raises(NotImplementedError):
        consensus.run_batch(V, [(np.ones((4, 257)), np.ones((257, 5)))], 3)
    with pytest.raises(ValueError):
        consensus.run_batch(V, starts, -1)


def test_restart_starts_follow_the_reference_draw_order():
    from nmf_rs import consensus

    V = np.arange(1.0, 13.0).reshape(3, 4)
    (W0, H0), (W1, _) = consensus.restart_starts(V, 2, 2)
    gen = np.random.default_rng(2024)
    s = float(np.sqrt(V.mean() / 2))
    np.testing.assert_array_equal(W0, gen.uniform(0, s, (3, 2)))
    np.testing.assert_array_equal(H0, gen.uniform(0, s, (2, 4)))
    np.testing.assert_array_equal(W1, np.random.default_rng(2025).uniform(0, s, (3, 2)))


def test_consensus_metrics():
    from nmf_rs import consensus

    H = np.array([[1.0, 0.9, 0.1, 0.0], [0.0, 0.1, 0.8, 1.0]])
    C = consensus.connectivity_matrix(H)
    np.testing.assert_array_equal(C, [[1, 1, 0, 0], [1, 1, 0, 0], [0, 0, 1, 1], [0, 0, 1, 1]])
    assert consensus.dispersion_coefficient(C) == 1.0
    assert consensus.cophenetic_correlation(C) == pytest.approx(1.0)
    assert consensus.dispersion_coefficient(np.full((4, 4), 0.5)) == 0.0
    H2 = np.array([[1.0, 0.0, 0.1, 0.0], [0.0, 0.1, 0.8, 1.0]])
    mixed = 0.5 * (C + consensus.connectivity_matrix(H2))
    assert 0.0 < consensus.dispersion_coefficient(mixed) < 1.0


def test_server_needs_a_device_and_checks_its_arguments():
    from nmf_rs import _native, serve

    import ctypes
    lib = _native.load()
    h = ctypes.c_void_p()
    assert lib.nmfcu_server_create(0, 0, 0, ctypes.byref(h)) == _native.INVALID_ARG
    assert lib.nmfcu_server_create(0, 4, -1, ctypes.byref(h)) == _native.INVALID_ARG
    if _native.device_count() == 0:
        with pytest.raises(RuntimeError):
            serve.Server(slots=2)


def test_cophenetic_is_the_coefficient_not_the_notebook_constant():
    from scipy.cluster.hierarchy import cophenet, linkage
    from scipy.spatial.distance import squareform

    from nmf_rs import consensus

    gen = np.random.default_rng(0)
    C = np.zeros((30, 30))
    for _ in range(10):
        lab = gen.integers(0, 3, 30)
        C += lab[:, None] == lab[None, :]
    C /= 10
    cond = squareform(1.0 - C, checks=False)
    expected = cophenet(linkage(cond, method="average"), cond)[0]
    assert consensus.cophenetic_correlation(C) == pytest.approx(expected, abs=1e-15)
    assert expected < 0.99


def test_batch_shape_setting_needs_no_gpu():
    # Selecting the batched kernel's shape is host state: it loads and
    # validates without a device.
    from nmf_rs import consensus
    n = consensus.batch_shape_count()
    assert n >= 1
    with pytest.raises(ValueError):
        consensus.set_batch_shape(n)
    with pytest.raises(ValueError):
        consensus.set_batch_shape(-2)
    consensus.set_batch_shape(0)
    consensus.set_batch_shape("auto")


def test_wide_rank_limits_checked_before_the_device():
    """Ranks above 32 run lee / brunet / hals / dnmf in FP64 up to
    NMFCU_MAX_WIDE_RANK; everything else is refused before any device work,
    so these raise on a machine without a GPU too."""
    V = np.ones((6, 7))
    W0, H0 = np.ones((6, 300)), np.ones((300, 7))
    with pytest.raises(NotImplementedError, match="largest supported rank"):
        _native.py_nmf_run("lee", V, W0, H0, 1)
    W0, H0 = np.ones((6, 40)), np.ones((40, 7))
    with pytest.raises(NotImplementedError, match="FP64 only"):
        _native.py_nmf_run("lee", V, W0, H0, 1, precision="fp32")
    for method in ("nsNMF", "ehals", "snmf/r"):
        with pytest.raises(NotImplementedError, match="run lee, brunet, hals and dnmf"):
            _native.py_nmf_run(method, V, W0, H0, 1)
