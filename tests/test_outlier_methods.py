"""The oracle's restatement of the reference's further outlier tests (local
sigma and divergence/vorticity, outlier_detection.py:246-381) against the
reference's own functions (tests/golden/outliers_ref.npz, written by
tests/golden/make_golden.py outliers).  The GPU kernels are checked against this
restatement in test_secondary_peaks_gpu.py."""

import os

import numpy as np

import ref_multipass as RM

GOLD = os.path.join(os.path.dirname(__file__), "golden", "outliers_ref.npz")


def test_sigma_and_divvort_restatement_equal_reference():
    z = np.load(GOLD)
    for k in range(int(z["n_cases"])):
        ux, uy = z[f"c{k}_ux"], z[f"c{k}_uy"]
        for thr in (1.5, 2.0, 3.0):
            assert np.array_equal(RM.sigma_flags(ux, uy, thr), z[f"c{k}_sigma_{thr}"]), (k, thr)
        assert np.array_equal(RM.divvort_flags(ux, uy), z[f"c{k}_divvort"]), k
        assert np.array_equal(RM.divvort_flags(ux, uy, 0.5, 0.7), z[f"c{k}_divvort_given"]), k
