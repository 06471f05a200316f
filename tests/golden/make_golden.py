"""Writes the golden fixtures of the quickstart known-answer tests.

Inputs: the matrix and starting point that omicverse/rust-NMF's own
``examples/tutorial_quickstart.ipynb`` builds (cells 1 and 3, from
``examples/build_notebooks.py:65-69, 81``): ``default_rng(0)``, 200 x 60,
rank 5, ``W_true, H_true ~ U(0.1, 1.5)``, ``+ U(0, 0.05)`` noise, and
``random_init(V, 5, seed=42)``.

Expected values: the reference's recorded outputs in that notebook
(the executed cells' text output), copied as numbers with their cell.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def quickstart_inputs():
    gen = np.random.default_rng(0)
    n, p, rank = 200, 60, 5
    w_true = gen.uniform(0.1, 1.5, (n, rank))
    h_true = gen.uniform(0.1, 1.5, (rank, p))
    V = w_true @ h_true + gen.uniform(0, 0.05, (n, p))
    init = np.random.default_rng(42)
    top = float(np.max(V))
    W0 = init.uniform(0.0, top, size=(n, rank))
    H0 = init.uniform(0.0, top, size=(rank, p))
    return V, W0, H0


KATS = {
    "source": "omicverse/rust-NMF examples/tutorial_quickstart.ipynb (executed outputs)",
    "V_min": 0.6152416663367443,            # cell 1
    "V_max": 8.061756004056358,             # cell 1
    "brunet_200_frob_norm": 9.11162723892749,   # cell 5: ||V - WH||_F, brunet, 200 it
    "lee_200_frob_norm_4dp": 8.0928,        # cell 7: lee, 200 it, printed to 4 d.p.
    "offset_200_frob_norm_4dp": 8.4113,     # cell 7: ||V - (WH + off)||_F, offset, 200 it
    "offset_200_range_2dp": [0.61, 2.21],   # cell 7: min / max of the final offsets
    "nsnmf_200_frob_norm_4dp": 30.8650,     # cell 7: ||V - WH||_F (fitted() omits S), nsNMF
    "brunet_stationary": {                  # cell 9
        "max_iter": 2000, "stationary_th": 1e-6, "check_interval": 10, "check_niter": 10,
        "n_iter": 2000, "final_kl": 0.5964519986834893, "n_deviances": 2001,
    },
    "single_step_brunet_delta_kl": 808788.7003988085,  # cell 13
}


def main():
    V, W0, H0 = quickstart_inputs()
    np.savez(HERE / "quickstart_inputs.npz", V=V, W0=W0, H0=H0)
    (HERE / "quickstart_kats.json").write_text(json.dumps(KATS, indent=2) + "\n")
    print("wrote", HERE / "quickstart_inputs.npz", HERE / "quickstart_kats.json")


if __name__ == "__main__":
    main()
