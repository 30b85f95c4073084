"""Host-side argument checks of the ensemble pass (pivtools_b200.ensemble), which
run before any device memory is touched: the reference's configuration rules
(pivtools_core/config.py ensemble properties, pivtools_core/validation.py:436-560)
as the GPU pass applies them."""

import numpy as np
import pytest

from pivtools_b200 import ensemble


def _make(**kw):
    args = dict(image_shape=(64, 64), window=(16, 16), overlap=75, window_type="square")
    args.update(kw)
    return ensemble.EnsemblePIV(**args)


def test_background_methods_and_refusals():
    assert set(ensemble._METHODS) == {"correlation", "correlation+dc_zero", "window_mean",
                                      "correlation+window_mean", "image", "image+window_mean", "image+dc_zero"}
    for name, (ms, bg, dc, two) in ensemble._METHODS.items():
        assert ms == ("window_mean" in name)
        assert bg == name.startswith("correlation")
        assert dc == name.endswith("dc_zero")
        assert two == name.startswith("image")
    with pytest.raises(ValueError, match="Invalid ensemble_background_subtraction_method"):
        _make(background="image+correlation")


def test_per_pair_normalisation_needs_window_mean():
    with pytest.raises(ValueError, match="per_pair_normalization"):
        _make(background="correlation+window_mean", per_pair_normalization=True)


def test_single_mode_refusals():
    with pytest.raises(ValueError, match="ensemble_type"):
        _make(runtype="double")
    with pytest.raises(ValueError, match="sum_window must be defined"):
        _make(window=(4, 4), runtype="single")
    with pytest.raises(ValueError, match="must be <="):
        _make(window=(4, 4), runtype="single", sum_window=(16, 16), fit_window=(20, 20))
    with pytest.raises(ValueError, match="must be >="):
        _make(window=(8, 8), runtype="single", sum_window=(4, 4))
    with pytest.raises(ValueError, match="square"):
        _make(window=(4, 4), runtype="single", sum_window=(16, 32))
    with pytest.raises(ValueError, match="belong to single mode"):
        _make(sum_window=(32, 32))


def test_pair_envelope_rules():
    w = np.ones((16, 16))
    e = ensemble.pair_envelope(w, w, (16, 16))
    assert e[8, 8] == 1.0 and np.all(e > 0)
    with pytest.raises(ValueError, match="share a shape"):
        ensemble.pair_envelope(np.ones((16, 16)), np.ones((8, 8)), (8, 8))
