"""CPU oracle for the NMF iteration loop -- TEST INFRASTRUCTURE ONLY.

A ctypes wrapper around ``liboracle.so`` (built from ``nmf_oracle.c`` by
``oracle/Makefile``), which restates the f64 loops of omicverse/rust-NMF
``rust/src/lib.rs`` (brunet :1529-1586, lee :1589-1647, offset :1650-1760,
nsNMF :1762-1830, hals :638-688, ehals :711-786, dnmf :827-906, lsNMF :945-1043, objectives :1410-1445,
stationary stop :1336-1401).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker / baseline.
The shipped library never calls it.

Parity status: pinned against the reference's recorded outputs in
``examples/tutorial_quickstart.ipynb`` (fixtures in ``tests/golden/``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle.so"
_lib = None

METHODS = {"brunet": 0, "lee": 1, "hals": 4, "ehals": 5, "dnmf": 6}
STOPS = {"max_iter": 0, "fixed": 0, "none": 0, "stationary": 1}

_i64 = ctypes.c_int64
_dp = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> Path:
    """Compile liboracle.so with the committed Makefile."""
    if force or not _LIB_PATH.exists() or (
        _LIB_PATH.stat().st_mtime < (_HERE / "nmf_oracle.c").stat().st_mtime
    ):
        subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def _cpu_fingerprint() -> str:
    """A short hash of this host's CPU model and feature flags."""
    import hashlib

    txt = ""
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith(("model name", "flags")):
                txt += ln
                if ln.startswith("flags"):
                    break
    except OSError:
        pass
    return hashlib.sha1(txt.encode()).hexdigest()[:12]


def use_native() -> Path:
    """Build (once per CPU model) and load a -march=native copy of the oracle
    for the CPU-baseline timing.  It computes the same values as the generic
    build: -ffp-contract=off and no fast-math hold in both."""
    global _lib, _LIB_PATH
    path = _HERE / f"liboracle_native_{_cpu_fingerprint()}.so"
    if not path.exists() or path.stat().st_mtime < (_HERE / "nmf_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(_HERE), "native", f"NATIVE_OUT={path}"],
                       check=True)
    _LIB_PATH = path
    _lib = None
    _load()
    return path


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        build()
    lib = ctypes.CDLL(str(_LIB_PATH))
    lib.orc_nmf_run.restype = ctypes.c_int
    lib.orc_nmf_run.argtypes = [
        ctypes.c_int, _i64, _i64, _i64, _dp, _dp, _dp, _i64, ctypes.c_double, ctypes.c_int,
        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
        ctypes.c_double, _i64, _i64, _dp, ctypes.POINTER(_i64), ctypes.POINTER(_i64),
        ctypes.c_int,
    ]
    for name in ("orc_update_h_brunet", "orc_update_w_brunet"):
        f = getattr(lib, name)
        f.restype = None
        f.argtypes = [_i64, _i64, _i64, _dp, _dp, _dp, _dp, ctypes.c_int]
    for name in ("orc_update_h_lee", "orc_update_w_lee"):
        f = getattr(lib, name)
        f.restype = None
        f.argtypes = [_i64, _i64, _i64, _dp, _dp, _dp, ctypes.c_double, _dp, ctypes.c_int]
    for name in ("orc_kl_divergence", "orc_euclidean_distance"):
        f = getattr(lib, name)
        f.restype = ctypes.c_double
        f.argtypes = [_i64, _i64, _i64, _dp, _dp, _dp]
    lib.orc_euclidean_distance_offset.restype = ctypes.c_double
    lib.orc_euclidean_distance_offset.argtypes = [_i64, _i64, _i64, _dp, _dp, _dp, _dp]
    lib.orc_nmf_run_nsnmf.restype = ctypes.c_int
    lib.orc_nmf_run_nsnmf.argtypes = [
        _i64, _i64, _i64, _dp, _dp, _dp, _i64, ctypes.c_double, ctypes.c_int, ctypes.c_double,
        _i64, _i64, _dp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.c_int,
    ]
    lib.orc_nmf_run_offset.restype = ctypes.c_int
    lib.orc_nmf_run_offset.argtypes = [
        _i64, _i64, _i64, _dp, _dp, _dp, _dp, _i64, ctypes.c_double, ctypes.c_int,
        ctypes.c_double, _i64, _i64, _dp, ctypes.POINTER(_i64), ctypes.POINTER(_i64),
        ctypes.c_int,
    ]
    lib.orc_weighted_distance.restype = ctypes.c_double
    lib.orc_weighted_distance.argtypes = [_i64, _i64, _i64, _dp, _dp, _dp, _dp]
    lib.orc_nmf_run_lsnmf.restype = ctypes.c_int
    lib.orc_nmf_run_lsnmf.argtypes = [
        _i64, _i64, _i64, _dp, _dp, _dp, _dp, _i64, ctypes.c_double, ctypes.c_int,
        ctypes.c_double, _i64, _i64, _dp, ctypes.POINTER(_i64), ctypes.POINTER(_i64),
        ctypes.c_int,
    ]
    lib.orc_fcnnls.restype = None
    lib.orc_fcnnls.argtypes = [ctypes.c_int, _i64, _dp, _dp, _i64, _i64, ctypes.c_double, _dp]
    lib.orc_cholesky.restype = ctypes.c_int
    lib.orc_cholesky.argtypes = [ctypes.c_int, _dp]
    lib.orc_nmf_run_snmf.restype = ctypes.c_int
    lib.orc_nmf_run_snmf.argtypes = [
        ctypes.c_int, _i64, _i64, _i64, _dp, _dp, _dp, _i64, ctypes.c_double, ctypes.c_double,
        ctypes.c_double, _dp, ctypes.c_int,
    ]
    if lib.orc_version() < 4:
        raise RuntimeError("liboracle.so is stale: rebuild it (make -C oracle)")
    _lib = lib
    return lib


def _c(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def nmf_run(method: str, V, W0, H0, max_iter: int, *, eps: float = 1e-9, rescale: bool = True,
            sparsity_h: float = 0.0, sparsity_w: float = 0.0, smoothness_h: float = 0.0,
            smoothness_w: float = 0.0, stop: str = "max_iter",
            stationary_th: float = 2.220446049250313e-16, check_interval: int = 50,
            check_niter: int = 10, num_threads: int | None = None) -> dict:
    """Oracle counterpart of ``py_nmf_run`` (lib.rs:1934-2169) for the four
    in-scope methods.  Returns ``{"W", "H", "n_iter", "deviances"}``."""
    lib = _load()
    V = _c(V)
    W = _c(W0).copy()
    H = _c(H0).copy()
    n, p = V.shape
    r = W.shape[1]
    dev = np.zeros(max(int(max_iter) + 1, 1), dtype=np.float64)
    nd = _i64(0)
    ni = _i64(0)
    rc = lib.orc_nmf_run(
        METHODS[method], n, p, r, _ptr(V), _ptr(W), _ptr(H), int(max_iter), float(eps),
        int(bool(rescale)), float(sparsity_h), float(sparsity_w), float(smoothness_h),
        float(smoothness_w), STOPS[stop.lower()], float(stationary_th), int(check_interval),
        int(check_niter), _ptr(dev), ctypes.byref(nd), ctypes.byref(ni),
        int(num_threads or os.cpu_count() or 1),
    )
    if rc == -2:
        raise ZeroDivisionError("stationary stop evaluated `iter % check_interval` with 0")
    if rc != 0:
        raise ValueError(f"oracle: unsupported method {method!r}")
    return {"W": W, "H": H, "n_iter": int(ni.value), "deviances": dev[: nd.value].copy()}


def _row_means_fwd(V: np.ndarray) -> np.ndarray:
    """rowMeans(V) with forward-order sums (the default offset, lib.rs:1667-1679)."""
    n, p = V.shape
    if p == 0:
        return np.full(n, np.nan)
    return np.cumsum(V, axis=1)[:, -1] / float(p)


def _stat_args(stop, stationary_th, check_interval, check_niter):
    return (STOPS[stop.lower()], float(stationary_th), int(check_interval), int(check_niter))


def nmf_nsnmf(V, W0, H0, max_iter: int, *, theta: float = 0.5, stop: str = "max_iter",
              stationary_th: float = 2.220446049250313e-16, check_interval: int = 50,
              check_niter: int = 10, num_threads: int | None = None) -> dict:
    """Oracle of ``py_nmf_run`` with method nsNMF (nmf_run_nsnmf, lib.rs:1762-1830)."""
    lib = _load()
    V = _c(V)
    W = _c(W0).copy()
    H = _c(H0).copy()
    n, p = V.shape
    r = W.shape[1]
    dev = np.zeros(max(int(max_iter) + 1, 1), dtype=np.float64)
    nd, ni = _i64(0), _i64(0)
    rc = lib.orc_nmf_run_nsnmf(
        n, p, r, _ptr(V), _ptr(W), _ptr(H), int(max_iter), float(theta),
        *_stat_args(stop, stationary_th, check_interval, check_niter), _ptr(dev),
        ctypes.byref(nd), ctypes.byref(ni), int(num_threads or os.cpu_count() or 1),
    )
    if rc == -2:
        raise ZeroDivisionError("stationary stop evaluated `iter % check_interval` with 0")
    return {"W": W, "H": H, "n_iter": int(ni.value), "deviances": dev[: nd.value].copy()}


def nmf_offset(V, W0, H0, max_iter: int, *, offset=None, eps: float = 1e-9,
               stop: str = "max_iter", stationary_th: float = 2.220446049250313e-16,
               check_interval: int = 50, check_niter: int = 10,
               num_threads: int | None = None) -> dict:
    """Oracle of ``py_nmf_run`` with method offset (nmf_run_offset, lib.rs:1650-1760).
    Returns ``{"W", "H", "offset", "n_iter", "deviances"}``."""
    lib = _load()
    V = _c(V)
    W = _c(W0).copy()
    H = _c(H0).copy()
    n, p = V.shape
    r = W.shape[1]
    off = _row_means_fwd(V) if offset is None else _c(offset).copy()
    if off.shape != (n,):
        raise ValueError(f"offset must have {n} entries")
    dev = np.zeros(max(int(max_iter) + 1, 1), dtype=np.float64)
    nd, ni = _i64(0), _i64(0)
    rc = lib.orc_nmf_run_offset(
        n, p, r, _ptr(V), _ptr(W), _ptr(H), _ptr(off), int(max_iter), float(eps),
        *_stat_args(stop, stationary_th, check_interval, check_niter), _ptr(dev),
        ctypes.byref(nd), ctypes.byref(ni), int(num_threads or os.cpu_count() or 1),
    )
    if rc == -2:
        raise ZeroDivisionError("stationary stop evaluated `iter % check_interval` with 0")
    return {"W": W, "H": H, "offset": off, "n_iter": int(ni.value),
            "deviances": dev[: nd.value].copy()}


def nmf_lsnmf(V, weight, W0, H0, max_iter: int, *, eps: float = 1e-9, stop: str = "max_iter",
              stationary_th: float = 2.220446049250313e-16, check_interval: int = 50,
              check_niter: int = 10, num_threads: int | None = None) -> dict:
    """Oracle of ``py_nmf_run`` with method lsnmf (nmf_run_lsnmf, lib.rs:945-1043)."""
    lib = _load()
    V, S = _c(V), _c(weight)
    W = _c(W0).copy()
    H = _c(H0).copy()
    n, p = V.shape
    if S.shape != V.shape:
        raise ValueError("weight must have V's shape")
    r = W.shape[1]
    dev = np.zeros(max(int(max_iter) + 1, 1), dtype=np.float64)
    nd, ni = _i64(0), _i64(0)
    rc = lib.orc_nmf_run_lsnmf(
        n, p, r, _ptr(V), _ptr(S), _ptr(W), _ptr(H), int(max_iter), float(eps),
        *_stat_args(stop, stationary_th, check_interval, check_niter), _ptr(dev),
        ctypes.byref(nd), ctypes.byref(ni), int(num_threads or os.cpu_count() or 1),
    )
    if rc == -2:
        raise ZeroDivisionError("stationary stop evaluated `iter % check_interval` with 0")
    return {"W": W, "H": H, "n_iter": int(ni.value), "deviances": dev[: nd.value].copy()}


def fcnnls(ctc, cta, eps: float = 0.0):
    """fcnnls (fcnnls.rs:297-470) on the normal equations ctc (l x l) and
    cta (l x P); returns K (l x P)."""
    lib = _load()
    ctc, cta = _c(ctc), _c(cta)
    l, P = cta.shape
    K = np.zeros((P, l))
    lib.orc_fcnnls(l, P, _ptr(ctc), _ptr(cta), P, 1, float(eps), _ptr(K))
    return K.T.copy()


def cholesky(a):
    lib = _load()
    f = _c(a).copy()
    ok = lib.orc_cholesky(f.shape[0], _ptr(f))
    return bool(ok), np.tril(f)


def nmf_snmf(V, W0, H0, max_iter: int, *, left: bool, eta: float = -1.0, beta: float = 0.01,
             eps: float = 1e-9, num_threads: int | None = None) -> dict:
    """Oracle of py_nmf_run with method snmf/r (left False) or snmf/l (left
    True): nmf_run_snmf_kim_park, lib.rs:1216-1320."""
    lib = _load()
    V = _c(V)
    W = _c(W0).copy()
    H = _c(H0).copy()
    n, p = V.shape
    k = W.shape[1]
    dev = np.zeros(max(int(max_iter), 1))
    rc = lib.orc_nmf_run_snmf(int(bool(left)), n, p, k, _ptr(V), _ptr(W), _ptr(H), int(max_iter),
                              float(eta), float(beta), float(eps), _ptr(dev),
                              int(num_threads or os.cpu_count() or 1))
    if rc != 0:
        raise ValueError("rank above 32")
    return {"W": W, "H": H, "n_iter": int(max_iter), "deviances": dev[: int(max_iter)].copy()}


def weighted_distance(V, weight, W, H) -> float:
    lib = _load()
    V, S, W, H = _c(V), _c(weight), _c(W), _c(H)
    return float(lib.orc_weighted_distance(V.shape[0], V.shape[1], W.shape[1], _ptr(V), _ptr(S),
                                           _ptr(W), _ptr(H)))


def nmf_method(method: str, V, W0, H0, max_iter: int, *, eps=1e-9, rescale=True,
               sparsity=0.01, smoothness=1.0, stop="max_iter", theta=0.5, offset=None,
               weight=None, **kw) -> dict:
    """Same as :func:`nmf_run` but with the Python-level routing of
    ``sparsity``/``smoothness`` that ``nmf()`` applies (python/nmf_rs/__init__.py:528-538):
    dnmf gets ``sparsity`` on both factors and no L2, the others get none.
    nsNMF and offset go to their own loops."""
    m = method.lower()
    if m in ("nsnmf", "ns", "ns_nmf"):
        return nmf_nsnmf(V, W0, H0, max_iter, theta=theta, stop=stop, **kw)
    if m == "offset":
        return nmf_offset(V, W0, H0, max_iter, offset=offset, eps=eps, stop=stop, **kw)
    if m in ("snmf/r", "snmf_r", "snmfr", "snmf/l", "snmf_l", "snmfl"):
        left = m in ("snmf/l", "snmf_l", "snmfl")
        # python/nmf_rs/__init__.py:528-538 -> lib.rs:2117-2148: snmf/r takes
        # beta = sparsity (on H), eta = smoothness (on W); snmf/l the mirror.
        return nmf_snmf(V, W0, H0, max_iter, left=left, eta=smoothness, beta=sparsity, eps=eps,
                        **kw)
    if m in ("lsnmf", "ls-nmf"):
        if weight is None:
            raise ValueError("method='lsnmf' requires a `weight` matrix of the same shape as V")
        return nmf_lsnmf(V, weight, W0, H0, max_iter, eps=eps, stop=stop, **kw)
    if method == "dnmf":
        sh = sw = float(sparsity)
    else:
        sh = sw = 0.0
    return nmf_run(method, V, W0, H0, max_iter, eps=eps, rescale=rescale, sparsity_h=sh,
                   sparsity_w=sw, smoothness_h=0.0, smoothness_w=0.0, stop=stop, **kw)


def update_h_brunet(V, W, H, num_threads=None):
    lib = _load()
    V, W, H = _c(V), _c(W), _c(H)
    out = np.empty_like(H)
    lib.orc_update_h_brunet(V.shape[0], V.shape[1], W.shape[1], _ptr(V), _ptr(W), _ptr(H),
                            _ptr(out), int(num_threads or os.cpu_count() or 1))
    return out


def update_w_brunet(V, W, H, num_threads=None):
    lib = _load()
    V, W, H = _c(V), _c(W), _c(H)
    out = np.empty_like(W)
    lib.orc_update_w_brunet(V.shape[0], V.shape[1], W.shape[1], _ptr(V), _ptr(W), _ptr(H),
                            _ptr(out), int(num_threads or os.cpu_count() or 1))
    return out


def update_h_lee(V, W, H, eps=1e-9, num_threads=None):
    lib = _load()
    V, W, H = _c(V), _c(W), _c(H)
    out = np.empty_like(H)
    lib.orc_update_h_lee(V.shape[0], V.shape[1], W.shape[1], _ptr(V), _ptr(W), _ptr(H),
                         float(eps), _ptr(out), int(num_threads or os.cpu_count() or 1))
    return out


def update_w_lee(V, W, H, eps=1e-9, num_threads=None):
    lib = _load()
    V, W, H = _c(V), _c(W), _c(H)
    out = np.empty_like(W)
    lib.orc_update_w_lee(V.shape[0], V.shape[1], W.shape[1], _ptr(V), _ptr(W), _ptr(H),
                         float(eps), _ptr(out), int(num_threads or os.cpu_count() or 1))
    return out


def kl_divergence(V, W, H) -> float:
    lib = _load()
    V, W, H = _c(V), _c(W), _c(H)
    return float(lib.orc_kl_divergence(V.shape[0], V.shape[1], W.shape[1], _ptr(V), _ptr(W),
                                       _ptr(H)))


def euclidean_distance(V, W, H) -> float:
    lib = _load()
    V, W, H = _c(V), _c(W), _c(H)
    return float(lib.orc_euclidean_distance(V.shape[0], V.shape[1], W.shape[1], _ptr(V),
                                            _ptr(W), _ptr(H)))


def euclidean_distance_offset(V, W, H, offset) -> float:
    lib = _load()
    V, W, H, off = _c(V), _c(W), _c(H), _c(offset)
    return float(lib.orc_euclidean_distance_offset(V.shape[0], V.shape[1], W.shape[1], _ptr(V),
                                                   _ptr(W), _ptr(H), _ptr(off)))
