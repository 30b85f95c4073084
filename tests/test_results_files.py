"""Result files: the .mat struct and the correlation-plane npz written by the
package's writers against the same files written by the reference's own writers
from the same per-pass fields (tests/golden/results_ref, made by
tests/golden/make_golden.py results)."""

import json
import os

import numpy as np
import pytest

from pivtools_b200 import results as R

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _result():
    d = np.load(os.path.join(GOLD, "results_in.npz"))
    res = R.PIVResult()
    for k in range(3):
        g = lambda key: d[f"p{k}_{key}"]
        ny, nx = g("ux").shape
        res.add_pass(R.PIVPassResult(
            n_windows=np.array([ny, nx], dtype=np.int32), ux_mat=g("ux"), uy_mat=g("uy"), nan_mask=g("nan_mask"),
            nan_reason=g("nan_reason"), peak_mag=g("peak_mag"), peak_ratio=g("peak_ratio"),
            peak_choice=g("peak_choice"), predictor_field=g("predictor"), b_mask=g("b_mask"),
            window_size=[int(v) for v in g("window_size")], win_ctrs_x=g("win_ctrs_x"), win_ctrs_y=g("win_ctrs_y"),
            debug_dump={"planes": g("planes"), "peak_finder": 3, "pk_loc_x_raw": g("pk_loc_x_raw"),
                        "pk_loc_y_raw": g("pk_loc_y_raw"), "pk_height_raw": g("peak_mag"),
                        "pk_ratio_raw": g("peak_ratio"), "sx": g("sx"), "sy": g("sy"), "sxy": g("sxy")}))
    return res


def _same(a, b, where):
    a, b = np.asarray(a), np.asarray(b)
    assert a.dtype == b.dtype and a.shape == b.shape, (where, a.dtype, b.dtype, a.shape, b.shape)
    if a.dtype.kind == "f":
        assert np.array_equal(a, b, equal_nan=True), where
    else:
        assert np.array_equal(a, b), where


def _load_struct(path):
    import scipy.io

    m = scipy.io.loadmat(path)
    assert [k for k in m if not k.startswith("__")] == ["piv_result"]
    return m["piv_result"]


@pytest.mark.parametrize("frame,kw", [(7, {}), (8, {"runs_to_save": [1, 2], "save_mode": "minimal"})])
def test_mat_struct_matches_reference_file(tmp_path, frame, kw):
    path = R.save_piv_result_distributed(_result(), tmp_path, frame, **kw)
    assert os.path.basename(path) == "B%05d.mat" % frame
    mine, ref = _load_struct(path), _load_struct(os.path.join(GOLD, "results_ref", "B%05d.mat" % frame))
    assert mine.dtype.names == ref.dtype.names and mine.shape == ref.shape
    for name in ref.dtype.names:
        for i in range(ref.shape[1]):
            _same(mine[name][0, i], ref[name][0, i], (frame, name, i))


def test_mat_struct_in_memory_types():
    st = R.piv_struct(_result())
    assert st.dtype.names[-1] == "nan_reason" and st["nan_reason"][0].dtype == np.int8
    assert st["ux"][0].dtype == np.float16 and st["peak_ratio"][0].dtype == np.float32
    assert st["ux"][0][0, 0] == np.float16(65504.0) and st["uy"][0][-1, -1] == np.float16(-65504.0)


def test_plane_dump_matches_reference_file(tmp_path):
    path = R.save_corr_plane_dump(_result(), tmp_path, 7)
    assert path.endswith(os.path.join("debug_corr_planes", "B00007_corrplanes.npz"))
    mine = np.load(path)
    ref = np.load(os.path.join(GOLD, "results_ref", "debug_corr_planes", "B00007_corrplanes.npz"))
    codes = sorted(int(c) for c in json.loads(str(mine["nan_reason_labels"])))
    assert codes == ref["nan_reason_label_codes"].tolist()
    assert set(mine.keys()) - {"nan_reason_labels", "pk_origin_note"} == set(ref.keys()) - {"nan_reason_label_codes"}
    for k in ref.keys():
        if k != "nan_reason_label_codes":
            _same(mine[k], ref[k], k)


def test_plane_dump_absent_without_planes(tmp_path):
    res = _result()
    for p in res.passes:
        p.debug_dump = None
    assert R.save_corr_plane_dump(res, tmp_path, 7) is None
