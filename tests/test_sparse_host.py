"""The sparse-V (CSR) entry point's host-side checks, CPU only: they run
before any device work, so a malformed CSR or an unsupported method is
refused with the reference's exception types on a machine without a GPU."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import nmf_rs
from nmf_rs import _native


def _call(indptr, indices, data, n, p, r=2, method="lee", **opts):
    o = _native.default_options()
    o.method = _native.parse_method(method)
    o.max_iter = 1
    for k, v in opts.items():
        setattr(o, k, v)
    indptr = np.ascontiguousarray(indptr, dtype=np.int64)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    data = np.ascontiguousarray(data, dtype=np.float64)
    W = np.ones((n, r))
    H = np.ones((r, p))
    nd, ni = ctypes.c_int64(0), ctypes.c_int64(0)
    _native.check(_native.load().nmfcu_run_csr(
        ctypes.byref(o), n, p, r, data.size, indptr.ctypes.data_as(_native._i64p),
        indices.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _native._ptr(data),
        _native._ptr(W), _native._ptr(H), _native._ptr(W), _native._ptr(H), None, 0,
        ctypes.byref(nd), ctypes.byref(ni)))


def test_bad_indptr_is_rejected():
    with pytest.raises(ValueError, match="indptr must start at 0"):
        _call([1, 2], [0, 1], [1.0, 2.0], 1, 3)
    with pytest.raises(ValueError, match="non-decreasing"):
        _call([0, 2, 1, 2], [0, 1], [1.0, 2.0], 3, 3)


def test_column_index_out_of_range_is_rejected():
    with pytest.raises(ValueError, match="outside"):
        _call([0, 1, 2], [0, 3], [1.0, 2.0], 2, 3)
    with pytest.raises(ValueError, match="outside"):
        _call([0, 1, 2], [0, -1], [1.0, 2.0], 2, 3)


def test_methods_other_than_the_four_are_unsupported():
    for method in ("offset", "nsNMF", "ehals", "snmf/r"):
        with pytest.raises(NotImplementedError, match="sparse"):
            _call([0, 1], [0], [1.0], 1, 2, method=method)


def test_reduced_precision_is_unsupported():
    with pytest.raises(NotImplementedError, match="FP64"):
        _call([0, 1], [0], [1.0], 1, 2, precision=_native.PRECISIONS["fp32"])


def test_python_route_checks_before_the_device():
    V = sp.random(20, 30, density=0.2, format="csr", random_state=0)
    with pytest.raises(NotImplementedError, match="needs a dense V"):
        nmf_rs.nmf(V, 3, "offset")
    neg = V.copy()
    neg.data[0] = -1.0
    with pytest.raises(ValueError, match="non-negative"):
        nmf_rs.nmf(neg, 3, "lee")


def test_csr_arrays_canonicalises():
    """Duplicates are summed and indices sorted before the library sees them
    (the library requires a canonical CSR)."""
    rows = np.array([0, 0, 1, 1, 1])
    cols = np.array([2, 0, 1, 1, 3])
    vals = np.array([1.0, 2.0, 3.0, 4.0, 5.0])
    V = sp.coo_matrix((vals, (rows, cols)), shape=(2, 4))
    indptr, indices, data, shape = _native.csr_arrays(V)
    assert shape == (2, 4)
    assert indptr.tolist() == [0, 2, 4]
    assert indices.tolist() == [0, 2, 1, 3]
    assert data.tolist() == [2.0, 1.0, 7.0, 5.0]
    assert indptr.dtype == np.int64 and indices.dtype == np.int32
