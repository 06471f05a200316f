"""Writes the NNDSVD golden fixtures: W0, H0 from omicverse/rust-NMF's own
``nndsvd_init`` (python/nmf_rs/__init__.py:129-219, pure Python over
scikit-learn's ``randomized_svd``), imported from the reference source tree.

The reference is only needed to regenerate the fixtures; the tests read the
committed ``nndsvd_cases.npz``.  scikit-learn version used: recorded in the
file as ``sklearn_version``.

Run from the repository root:
    python tests/golden/make_nndsvd_golden.py /path/to/rust-NMF
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(ROOT / "rust-nmf_b200"))

import make_golden  # noqa: E402
from nmf_rs import synthetic  # noqa: E402

# name: (V builder, rank, fill, seed, n_oversamples)
CASES = {
    # n >= p, 7 power iterations (rank < 0.1 min(n, p))
    "quickstart_mean": (lambda: make_golden.quickstart_inputs()[0], 5, "mean", 0, 10),
    "quickstart_zero": (lambda: make_golden.quickstart_inputs()[0], 5, "zero", 3, 10),
    # n < p (the SVD of V^T), 4 power iterations
    "wide_eps": (lambda: synthetic.counts_matrix(60, 300, 6, 0.3, seed=7), 8, "eps", 1, 10),
    # more test vectors than rows: the LU factors narrow to 12 columns.  No
    # all-zero row: the singular vectors' entries on such a row are rounding
    # noise whose sign decides between the mean fill and ~1e-16.
    "tiny_mean": (lambda: synthetic.counts_matrix(12, 40, 3, 0.3, seed=9) + 0.01, 4, "mean", 2,
                  10),
    # rank 30 + 10 oversamples: two column chunks of the device product
    "rank30_mean": (lambda: synthetic.counts_matrix(150, 120, 12, 0.3, seed=5), 30, "mean", 4,
                    10),
}


def main(reference: str):
    import importlib.util

    import sklearn

    spec = importlib.util.spec_from_file_location(
        "ref_nmf_rs", Path(reference) / "python" / "nmf_rs" / "__init__.py")
    ref = importlib.util.module_from_spec(spec)
    sys.modules["ref_nmf_rs"] = ref
    spec.loader.exec_module(ref)
    out = {"sklearn_version": np.array(sklearn.__version__)}
    for name, (build, rank, fill, seed, over) in CASES.items():
        V = build()
        W, H = ref.nndsvd_init(V, rank, fill=fill, seed=seed, n_oversamples=over)
        if not name.startswith("quickstart"):  # quickstart V is in quickstart_inputs.npz
            out[f"{name}__V"] = V
        out[f"{name}__W"] = W
        out[f"{name}__H"] = H
        out[f"{name}__meta"] = np.array([rank, seed, over])
        out[f"{name}__fill"] = np.array(fill)
    np.savez_compressed(HERE / "nndsvd_cases.npz", **out)
    print("wrote", HERE / "nndsvd_cases.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_nndsvd_golden.py <path of the reference checkout>")
    main(sys.argv[1])
