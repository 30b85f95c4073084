"""Per-pass results of the instantaneous path and the reference's result files.

PIVPassResult / PIVResult carry the fields of the reference's per-pass record
(pivtools_cli/piv/piv_result.py:8-46) for one image pair; `MultipassPIV.collect`
fills them from the device buffers of a batch step.  Two writers produce the
reference's files from them:

  save_piv_result_distributed  one `B%05d.mat` per pair holding the `piv_result`
                               struct array, one element per pass
                               (pivtools_cli/piv/save_results.py:23-85, :790-946);
  save_corr_plane_dump         the correlation-plane npz next to it, when the
                               step kept its planes (save_results.py:88-172).

The struct layout, field names, dtypes and the float16 clamp are the reference's
file format, kept identical so that its readers and post-processing load these
files unchanged.
"""

from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

# Invalid-vector reason codes (pivtools_cli/piv/piv_backend/nan_reason_codes.py:18-25)
NAN_MASKED = -1
NAN_VALID = 0
NAN_FIT_FAIL = 1
NAN_LARGE_DISP = 6
NAN_UNCLASSIFIED = 9
NAN_OUTLIER = 10
NAN_SECONDARY_OUTLIER = 12
NAN_PEAK_MAG_NAN = 13

NAN_REASON_LABELS = {
    NAN_MASKED: "window masked",
    NAN_VALID: "valid vector",
    NAN_FIT_FAIL: "peak fit failed (no peak found or fit not converged)",
    NAN_LARGE_DISP: "displacement beyond the pass's gate",
    NAN_UNCLASSIFIED: "invalid, claimed by no stage",
    NAN_OUTLIER: "outlier test on the primary peak",
    NAN_SECONDARY_OUTLIER: "outlier test on a substituted secondary peak",
    NAN_PEAK_MAG_NAN: "peak height of the chosen peak is NaN",
}

FLOAT16_MAX = 65504.0

# Field order of the full-mode struct (save_results.py:837-852)
_FULL_FIELDS = ("ux", "uy", "b_mask", "nan_mask", "win_ctrs_x", "win_ctrs_y", "peak_mag", "peak_ratio",
                "peak_choice", "n_windows", "predictor_field", "window_size", "nan_reason")
_MINIMAL_FIELDS = ("ux", "uy", "b_mask")


@dataclass
class PIVPassResult:
    """One pass of one pair (piv_result.py:8-28); arrays are host NumPy arrays."""
    n_windows: Optional[np.ndarray] = None          # int32 [n_win_y, n_win_x]
    ux_mat: Optional[np.ndarray] = None             # float32 (n_win_y, n_win_x), infilled, 0 at masked
    uy_mat: Optional[np.ndarray] = None
    nan_mask: Optional[np.ndarray] = None           # bool, invalid or masked
    peak_mag: Optional[np.ndarray] = None           # float32 (n_peaks, n_win_y, n_win_x), NaN where gated
    peak_ratio: Optional[np.ndarray] = None         # float32 (n_win_y, n_win_x), primary / second peak
    peak_choice: Optional[np.ndarray] = None        # int (n_win_y, n_win_x): 1 = primary peak used, 0 = invalid
    predictor_field: Optional[np.ndarray] = None    # float32 (n_win_y, n_win_x, 2) = [dy, dx]
    primary_peak_mag: Optional[np.ndarray] = None
    b_mask: Optional[np.ndarray] = None             # bool (n_win_y, n_win_x)
    window_size: Optional[tuple] = None
    win_ctrs_x: Optional[np.ndarray] = None
    win_ctrs_y: Optional[np.ndarray] = None
    nan_reason: Optional[np.ndarray] = None         # int8 codes above
    debug_dump: Optional[dict] = None               # correlation-plane payload (never in the .mat)


@dataclass
class PIVResult:
    """All passes of one pair (piv_result.py:31-46)."""
    passes: List[PIVPassResult] = field(default_factory=list)

    def add_pass(self, pass_result: PIVPassResult):
        self.passes.append(pass_result)


def to_half(arr):
    """float16 copy of a float array, clamped to the float16 range with NaN kept
    (save_results.py:1066-1097); other dtypes and empty arrays pass unchanged."""
    if arr is None or arr.size == 0 or arr.dtype.kind != "f":
        return arr
    out = np.clip(arr, -FLOAT16_MAX, FLOAT16_MAX)
    out = np.where(np.isnan(arr), np.nan, out)
    return out.astype(np.float16)


def piv_struct(piv_result: PIVResult, runs_to_save=None, save_mode: str = "full") -> np.ndarray:
    """The `piv_result` struct array, one element per pass; passes outside
    runs_to_save hold empty (0, 0) arrays (save_results.py:790-946)."""
    names = _MINIMAL_FIELDS if save_mode == "minimal" else _FULL_FIELDS
    n = len(piv_result.passes)
    st = np.empty((n,), dtype=[(k, object) for k in names])
    first = piv_result.passes[0]
    ddt = first.ux_mat.dtype if (first.ux_mat is not None and first.ux_mat.size > 0) else np.float64
    empty = np.empty((0, 0), dtype=ddt)
    for i in range(n):
        for k in names:
            st[k][i] = empty
    runs = list(range(n)) if runs_to_save is None else list(runs_to_save)
    for i, pr in enumerate(piv_result.passes):
        if i not in runs:
            continue
        if pr.ux_mat is not None:
            st["ux"][i] = to_half(pr.ux_mat)
        if pr.uy_mat is not None:
            st["uy"][i] = to_half(pr.uy_mat)
        if pr.b_mask is not None:
            st["b_mask"][i] = pr.b_mask
        elif pr.nan_mask is not None:
            st["b_mask"][i] = pr.nan_mask
        if save_mode == "minimal":
            continue
        if pr.nan_mask is not None:
            st["nan_mask"][i] = pr.nan_mask
        if pr.nan_reason is not None:
            st["nan_reason"][i] = pr.nan_reason
        for k in ("win_ctrs_x", "win_ctrs_y", "peak_mag"):
            v = getattr(pr, k)
            if v is not None:
                st[k][i] = to_half(v)
        if pr.peak_ratio is not None:
            st["peak_ratio"][i] = pr.peak_ratio.astype(np.float32, copy=False)
        if pr.peak_choice is not None:
            st["peak_choice"][i] = pr.peak_choice
        if pr.n_windows is not None:
            st["n_windows"][i] = pr.n_windows
        if pr.predictor_field is not None:
            st["predictor_field"][i] = to_half(pr.predictor_field)
        if pr.window_size is not None:
            st["window_size"][i] = pr.window_size
    return st


def save_piv_result_distributed(piv_result: PIVResult, output_path, frame_number: int, runs_to_save=None,
                                vector_fmt: str = "B%05d.mat", save_mode: str = "full",
                                do_compression: bool = True) -> str:
    """Write one pair's passes to output_path / (vector_fmt % frame_number) as
    {"piv_result": struct} (save_results.py:23-85).  Returns the path."""
    import scipy.io

    os.makedirs(output_path, exist_ok=True)
    filename = os.path.join(str(output_path), vector_fmt % frame_number)
    if len(piv_result.passes) == 0:
        return filename
    scipy.io.savemat(filename, {"piv_result": piv_struct(piv_result, runs_to_save, save_mode)}, oned_as="row",
                     do_compression=do_compression)
    return filename


_DUMP_KEYS = ("planes", "pk_loc_x_raw", "pk_loc_y_raw", "pk_height_raw", "pk_ratio_raw", "sx", "sy", "sxy",
              "peak_finder")


def save_corr_plane_dump(piv_result: PIVResult, output_path, frame_number: int,
                         vector_fmt: str = "B%05d.mat") -> Optional[str]:
    """Write output_path/debug_corr_planes/<stem>_corrplanes.npz with every pass's
    correlation planes, raw peak outputs and validated fields under `pass<k>_`
    keys (save_results.py:88-172); None when no pass kept its planes."""
    if not any(p.debug_dump is not None for p in piv_result.passes):
        return None
    ddir = os.path.join(str(output_path), "debug_corr_planes")
    os.makedirs(ddir, exist_ok=True)
    stem = os.path.splitext(vector_fmt % frame_number)[0]
    filename = os.path.join(ddir, f"{stem}_corrplanes.npz")
    payload = {
        "frame_number": np.int64(frame_number),
        "n_passes": np.int64(len(piv_result.passes)),
        "nan_reason_labels": json.dumps({str(k): v for k, v in NAN_REASON_LABELS.items()}),
        "pk_origin_note": ("peak pixel of a plane = (pk_loc_y_raw + H//2, pk_loc_x_raw + W//2); planes are the "
                           "raw correlation the peak search saw; an all-zero plane is a skipped window"),
    }
    for k, pr in enumerate(piv_result.passes):
        dd = pr.debug_dump
        if dd is None:
            continue
        pre = f"pass{k}_"
        for key in _DUMP_KEYS:
            payload[pre + key] = dd[key]
        payload[pre + "ux"] = pr.ux_mat
        payload[pre + "uy"] = pr.uy_mat
        payload[pre + "nan_mask"] = pr.nan_mask
        payload[pre + "nan_reason"] = pr.nan_reason
        payload[pre + "peak_choice"] = pr.peak_choice
        payload[pre + "b_mask"] = pr.b_mask
        payload[pre + "predictor"] = pr.predictor_field
        payload[pre + "win_ctrs_x"] = pr.win_ctrs_x
        payload[pre + "win_ctrs_y"] = pr.win_ctrs_y
        payload[pre + "window_size"] = np.asarray(pr.window_size)
    np.savez_compressed(filename, **payload)
    return filename
