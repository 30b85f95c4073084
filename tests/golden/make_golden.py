"""Generate the golden fixtures from the reference itself.

Run in a container that has the reference sources (it reads them only through
the reference-compiled libraries `oracle/_ref/*.so`, built by
`make -C oracle ref`, and, for the k-space fixture, by importing the reference's
Python package).  The fixtures are committed; tests never need the reference.

    python tests/golden/make_golden.py            # peakfit_ref.npz, warp_ref.npz
    python tests/golden/make_golden.py kspace     # kspace_ref.npz
    python tests/golden/make_golden.py kspace_c   # kspace_c_ref.npz (compiled k-space fitter)
    python tests/golden/make_golden.py ensemble   # ensemble_ref.npz
    python tests/golden/make_golden.py ingest     # ingest_ref.npz
    python tests/golden/make_golden.py validate   # validate_ref.npz
    python tests/golden/make_golden.py results    # results_in.npz, results_ref/
    python tests/golden/make_golden.py floor      # floor_ref.npz
    python tests/golden/make_golden.py vmask      # vmask_ref.npz
    python tests/golden/make_golden.py infill     # infill_ref.npz
    python tests/golden/make_golden.py xcorr      # xcorr_ref.npz, triple_ref.npz
    python tests/golden/make_golden.py lavision   # lavision_ref.npz
    python tests/golden/make_golden.py pfill      # pfill_ref.npz
    python tests/golden/make_golden.py outliers   # outliers_ref.npz

The reference checkout is named by $PIVTOOLS_REF (its libraries are built from it
by `make -C oracle ref PIVTOOLS_REF=...`).
"""

from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

REF_ROOT = os.environ.get("PIVTOOLS_REF", "")
if not os.path.isdir(os.path.join(REF_ROOT, "pivtools_cli")):
    raise SystemExit("set PIVTOOLS_REF to the reference checkout")
sys.path.insert(0, os.path.join(ROOT, "python-pivtools_b200"))
sys.path.insert(0, HERE)


def gauss(shape, amp, i0, j0, s1, s2, cov, kind):
    h, w = shape
    ii, jj = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
    y = ii - (h - 1) / 2 - i0
    x = jj - (w - 1) / 2 - j0
    if kind == 4:
        z = amp * np.exp(-(y * y + x * x) / (s1 * s1))
    elif kind == 5:
        z = amp * np.exp(-(y * y / (s1 * s1) + x * x / (s2 * s2)))
    else:
        z = amp * np.exp(-0.5 * (y * y / s1 + x * x / s2 + 2.0 * y * x * cov))
    return z.astype(np.float32)


def peakfit_cases():
    """Planes of the reference's own peak-fit tests (test_instantaneous_peaks.py,
    test_peakfit_batch.py) plus a seeded noisy battery with plane weights."""
    cases = []   # (plane, fit_type, n_peaks, weight or None)
    for shape in [(17, 17), (33, 33), (65, 65), (33, 65)]:
        for disp in [(0.0, 0.0), (0.35, 0.27), (0.1, -0.4)]:
            for t in (3, 4, 5, 6):
                if t in (3, 4):
                    p = gauss(shape, 1000.0, *disp, 1.5, 1.5, 0.0, 4)
                elif t == 5:
                    p = gauss(shape, 1000.0, *disp, 1.5, 1.5, 0.0, 5)
                else:
                    p = gauss(shape, 1000.0, *disp, 2.25, 2.25, 0.0, 6)
                cases.append((p, t, 1, None))
    for t in (4, 5, 6):
        for sr, sc in [(1.5, 1.5), (1.5, 2.0), (1.0, 3.0)]:
            if t == 4:
                s = np.sqrt((sr * sr + sc * sc) / 2)
                p = gauss((33, 33), 1000.0, 0.35, 0.27, s, s, 0.0, 4)
            elif t == 5:
                p = gauss((33, 33), 1000.0, 0.35, 0.27, sr, sc, 0.0, 5)
            else:
                p = gauss((33, 33), 1000.0, 0.35, 0.27, sr * sr, sc * sc, 0.0, 6)
            cases.append((p, t, 1, None))
    ell = gauss((33, 33), 1000.0, 0.35, 0.27, 1.5, 2.5, 0.0, 5)
    for t in (3, 4, 5, 6):
        cases.append((ell, t, 1, None))
    # failure sentinels
    z = np.zeros((33, 33), np.float32)
    ramp = (np.arange(33, dtype=np.float32)[:, None] * np.ones(33, np.float32)[None, :]) + 1.0
    poison = gauss((33, 33), 1000.0, 0.0, 0.0, 1.5, 1.5, 0.0, 4)
    poison[17, 17] = np.nan
    spike = np.random.RandomState(0).uniform(0.0, 1.0, (33, 33)).astype(np.float32)
    spike[16, 16] = 2.0
    for t in (3, 4, 5, 6):
        for p in (z, ramp, poison, spike):
            cases.append((p, t, 1, None))
    # seeded noisy battery, with and without a compensation weight, 1 and 3 peaks
    rng = np.random.default_rng(20261203)
    for k in range(72):
        t = (3, 4, 5, 6)[k % 4]
        kind = 4 if t == 3 else t
        s1, s2 = rng.uniform(1.0, 2.5, 2)
        if kind == 6:
            s1, s2 = s1 * s1, s2 * s2
        p = gauss((33, 33), rng.uniform(100, 1000), *rng.uniform(-0.45, 0.45, 2), s1, s2,
                  rng.uniform(-0.2, 0.2) / np.sqrt(s1 * s2), kind)
        p = (p + rng.normal(0.0, rng.choice([0.0, 2.0, 10.0]), p.shape)).astype(np.float32)
        wt = (1.0 + 0.2 * rng.random((33, 33))).astype(np.float32) if k % 3 == 0 else None
        cases.append((p, t, 3 if k % 9 == 0 else 1, wt))
    return cases


def make_peakfit():
    R = O.ref_peakfit()
    if R is None:
        raise SystemExit("oracle/_ref/libpeakfit_ref.so missing: run `make -C oracle ref`")
    cases = peakfit_cases()
    shapes = sorted({c[0].shape for c in cases})
    out = {"shapes": np.array(shapes, np.int32)}
    for si, shape in enumerate(shapes):
        sel = [c for c in cases if c[0].shape == shape]
        planes = np.stack([c[0] for c in sel]).astype(np.float32)
        types = np.array([c[1] for c in sel], np.int32)
        npk = np.array([c[2] for c in sel], np.int32)
        has_w = np.array([c[3] is not None for c in sel], bool)
        weights = np.stack([c[3] if c[3] is not None else np.ones(shape, np.float32) for c in sel])
        loc = np.full((len(sel), 9), np.nan, np.float32)
        sd = np.full((len(sel), 9), np.nan, np.float32)
        ratio = np.zeros(len(sel), np.float32)
        N = np.array(shape, np.int32)
        for k, (p, t, m, w) in enumerate(sel):
            l = np.zeros(3 * m, np.float32)
            s = np.zeros(3 * m, np.float32)
            R.lsqpeaklocate_lm(np.ascontiguousarray(p), N, l, m, t, s,
                               None if w is None else np.ascontiguousarray(w).ctypes.data)
            loc[k, :3 * m] = l
            sd[k, :3 * m] = s
            ratio[k] = R.peak_detectability(np.ascontiguousarray(p), N)
        out[f"s{si}_planes"] = planes
        out[f"s{si}_types"] = types
        out[f"s{si}_npeaks"] = npk
        out[f"s{si}_hasw"] = has_w
        out[f"s{si}_weights"] = weights.astype(np.float32)
        out[f"s{si}_loc"] = loc
        out[f"s{si}_sd"] = sd
        out[f"s{si}_ratio"] = ratio
    # batch route (reference lockstep fitter; 8 lanes as the reference library is compiled here)
    W = R.peakfit_batch_lanes()
    rng = np.random.default_rng(7)
    bplanes, btypes, bloc, bsd = [], [], [], []
    for t in (4, 5, 6):
        for rep in range(3):
            pl = []
            for _ in range(W):
                s1, s2 = rng.uniform(1.0, 2.5, 2)
                if t == 6:
                    s1, s2 = s1 * s1, s2 * s2
                p = gauss((33, 33), rng.uniform(100, 1000), *rng.uniform(-0.45, 0.45, 2), s1, s2,
                          rng.uniform(-0.2, 0.2) / np.sqrt(s1 * s2), t)
                pl.append((p + rng.normal(0.0, 3.0, p.shape)).astype(np.float32))
            pl = np.stack(pl)
            l = np.zeros(3 * W, np.float32)
            s = np.zeros(3 * W, np.float32)
            R.lsqpeaklocate_lm_batch(pl, W, np.array([33, 33], np.int32), t, l, s, None)
            bplanes.append(pl)
            btypes.append(np.full(W, t, np.int32))
            bloc.append(l.reshape(3, W).T)
            bsd.append(s.reshape(3, W).T)
    out["batch_planes"] = np.concatenate(bplanes)
    out["batch_types"] = np.concatenate(btypes)
    out["batch_loc"] = np.concatenate(bloc)
    out["batch_sd"] = np.concatenate(bsd)
    np.savez_compressed(os.path.join(HERE, "peakfit_ref.npz"), **out)
    print("peakfit_ref.npz:", sum(v.nbytes for v in out.values()), "bytes raw")


def make_warp():
    RW = O.ref_warp()
    if RW is None:
        raise SystemExit("oracle/_ref/libfusedwarp_ref.so missing: run `make -C oracle ref`")
    RW.fused_warp_set_impl(0)
    rng = np.random.default_rng(11)
    N, H, W = 2, 48, 64
    ia = rng.uniform(0, 255, (N, H, W)).astype(np.float32)
    ib = rng.uniform(0, 255, (N, H, W)).astype(np.float32)
    cy = np.linspace(-4.5, H + 3.5, 8).astype(np.float32)
    cx = np.linspace(-4.5, W + 3.5, 10).astype(np.float32)
    pdy = rng.normal(0, 2.5, (N, 8, 10)).astype(np.float32)
    pdx = rng.normal(0, 2.5, (N, 8, 10)).astype(np.float32)
    out = dict(imgs_a=ia, imgs_b=ib, ctrs_y=cy, ctrs_x=cx, pred_dy=pdy, pred_dx=pdx)
    for mode in (0, 1):
        for rs in (0, 1):
            ra = np.zeros_like(ia)
            rb = np.zeros_like(ib)
            RW.fused_symmetric_warp_batch(ia, ib, ra, rb, pdy, pdx, N, H, W, 8, 10, cy, cx, mode, 0, rs)
            out[f"out_a_m{mode}_r{rs}"] = ra
            out[f"out_b_m{mode}_r{rs}"] = rb
    # the reference's default SIMD route (AVX2 interior association as compiled here)
    RW.fused_warp_set_impl(1)
    for mode in (0, 1):
        ra = np.zeros_like(ia)
        rb = np.zeros_like(ib)
        RW.fused_symmetric_warp_batch(ia, ib, ra, rb, pdy, pdx, N, H, W, 8, 10, cy, cx, mode, 0, 0)
        out[f"simd_a_m{mode}"] = ra
        out[f"simd_b_m{mode}"] = rb
    RW.fused_warp_set_impl(0)
    np.savez_compressed(os.path.join(HERE, "warp_ref.npz"), **out)
    print("warp_ref.npz written")


def make_kspace():
    """Fixtures from the reference's NumPy k-space oracle (fit_windows_kspace_lm_numpy,
    pivtools_cli/piv/piv_backend/kspace_lm_fitting.py:964) on its own test batch
    generator (unit-tests/synthetic_correlations.py)."""
    sys.path.insert(0, REF_ROOT)
    sys.path.insert(0, os.path.join(REF_ROOT, "unit-tests"))
    from synthetic_correlations import generate_correlation_triplet, make_mock_config

    from pivtools_cli.piv.piv_backend.kspace_lm_fitting import fit_windows_kspace_lm_numpy

    corr = (24, 24)
    n = 24
    rng = np.random.default_rng(7)
    aa, bb, ab = [], [], []
    for i in range(n):
        A, B, C = generate_correlation_triplet(
            corr, sigma_particle_x=1.8 + 0.4 * rng.random(), sigma_particle_y=1.8 + 0.4 * rng.random(),
            sigma_stress_xx=0.3 * rng.random(), sigma_stress_yy=0.3 * rng.random(),
            mu_x=rng.uniform(-1.5, 1.5), mu_y=rng.uniform(-1.5, 1.5), noise_std=0.002, seed=100 + i)
        aa.append(A.ravel())
        bb.append(B.ravel())
        ab.append(C.ravel())
    mask = np.zeros(n, bool)
    mask[::7] = True
    R_AA, R_BB, R_AB = (np.concatenate(x) for x in (aa, bb, ab))
    ky, kx = np.meshgrid(np.linspace(-1, 1, corr[0]), np.linspace(-1, 1, corr[1]), indexing="ij")
    P = np.tile((1.0 + 0.6 * np.exp(-(kx ** 2 + ky ** 2) / 0.25)).ravel(), n)
    out = dict(R_AA=R_AA, R_BB=R_BB, R_AB=R_AB, mask=mask, P_win=P, corr=np.array(corr))
    for shape in ("gaussian", "kx4", "ky4", "kx4+ky4"):
        for floor in ("flat", "coloured"):
            cfg = make_mock_config(ensemble_kspace_shape=shape, ensemble_kspace_floor=floor)
            kw = {"P_win": P} if floor == "coloured" else {}
            g, s, ig, diag = fit_windows_kspace_lm_numpy(R_AA, R_BB, R_AB, mask, corr, cfg, 0,
                                                          return_diagnostics=True, **kw)
            key = f"{shape}_{floor}"
            out[f"{key}_gauss"] = np.asarray(g)
            out[f"{key}_status"] = np.asarray(s)
            out[f"{key}_init"] = np.asarray(ig)
    np.savez_compressed(os.path.join(HERE, "kspace_ref.npz"), **out)
    print("kspace_ref.npz written")


def make_kspace_c():
    """Outputs of the reference's compiled kspace_lm_fit_batch (kspace_lm_fit.c,
    built by make -C oracle ref) on kspace_ref.npz's inputs."""
    g = np.load(os.path.join(HERE, "kspace_ref.npz"))
    if O.ref_kspace() is None:
        raise SystemExit("build the reference k-space fitter first: make -C oracle ref")
    corr = tuple(int(v) for v in g["corr"])
    out = {}
    for shape in ("gaussian", "kx4", "ky4", "kx4+ky4"):
        for floor in ("flat", "coloured"):
            o = O.ref_kspace_fit(g["R_AA"], g["R_BB"], g["R_AB"], g["mask"], corr,
                                 use_kx4=int("kx4" in shape), use_ky4=int("ky4" in shape),
                                 P_win=g["P_win"] if floor == "coloured" else None, n_threads=1)
            assert o["ret"] == 0
            key = f"{shape}_{floor}"
            for k in ("gauss_flat", "status", "initial_guess", "gain", "N0", "iters"):
                out[f"{key}_{k}"] = o[k]
    np.savez_compressed(os.path.join(HERE, "kspace_c_ref.npz"), **out)
    print("kspace_c_ref.npz written")


def _reference_functions(path, names):
    """Compile the named module-level functions of a reference source file on
    their own (they need only NumPy; the module's other imports are not
    available here)."""
    import ast

    tree = ast.parse(open(path).read())
    body = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    ns = {"np": np}
    exec(compile(ast.Module(body=body, type_ignores=[]), path, "exec"), ns)
    return [ns[n] for n in names]


def make_ensemble():
    """Fixtures for the ensemble finalise steps, from the reference's own
    functions (pivtools_cli/piv/piv_backend/single_pass_accumulator.py:52-125):
    the linear pair-count envelope and the per-window plane-mean removal."""
    sys.path.insert(0, os.path.join(ROOT, "python-pivtools_b200"))
    from pivtools_b200 import geometry

    env_fn, dc_fn = _reference_functions(
        os.path.join(REF_ROOT, "pivtools_cli/piv/piv_backend/single_pass_accumulator.py"),
        ["_linear_pair_envelope", "_zero_plane_means"])
    out = {}
    for wtype in ("square", "gaussian", "blackman"):
        for n in (16, 32):
            w = geometry.window_weight((n, n), wtype).astype(np.float64)
            out[f"w_{wtype}_{n}"] = w
            out[f"env_{wtype}_{n}"] = env_fn(w, w, (n, n))
    rng = np.random.default_rng(11)
    planes = rng.standard_normal(7 * 16 * 16).astype(np.float32) + 3.0
    out["dc_in"] = planes
    out["dc_out"] = dc_fn(planes.copy(), 7, (16, 16))
    # single mode: the reference's grid and padding (window_utils.py), its
    # singlepix / bsingle weights (base.py:_window_weight_fun, a static method
    # compiled here on its own) and the envelopes the finalise divides by
    import ast
    import importlib.util

    spec = importlib.util.spec_from_file_location("ref_window_utils",
                                                  os.path.join(REF_ROOT, "pivtools_core/window_utils.py"))
    wu = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wu)
    base = os.path.join(REF_ROOT, "pivtools_cli/piv/piv_backend/base.py")
    tree = ast.parse(open(base).read())
    fn = [m for c in tree.body if isinstance(c, ast.ClassDef) for m in c.body
          if isinstance(m, ast.FunctionDef) and m.name == "_window_weight_fun"][0]
    fn.decorator_list = []
    ns = {"np": np}
    exec(compile(ast.Module(body=[fn], type_ignores=[]), base, "exec"), ns)
    wfun = ns["_window_weight_fun"]
    cases = [((512, 384), (4, 4), (16, 16), 50), ((300, 257), (6, 4), (17, 15), 75), ((128, 160), (8, 8), (32, 32), 0),
             ((256, 256), (1, 1), (16, 16), 50)]
    for k, (shape, win, sumw, ov) in enumerate(cases):
        r = wu.compute_window_centers_single_mode(shape, win, sumw, ov)
        out[f"single{k}_cx"], out[f"single{k}_cy"] = r.win_ctrs_x, r.win_ctrs_y
        out[f"single{k}_meta"] = np.array([r.n_win_x, r.n_win_y, r.win_spacing_x, r.win_spacing_y, *r.padding])
        out[f"single{k}_case"] = np.array([*shape, *win, *sumw, ov])
    for win, sumw, fit in (((4, 4), (16, 16), (16, 16)), ((8, 8), (32, 32), (24, 24)), ((5, 5), (16, 16), (12, 12))):
        wa = wfun(win, "singlepix", sumw)
        wb = wfun(sumw, "bsingle", sumw)
        key = f"sp_{win[0]}_{sumw[0]}_{fit[0]}"
        out[key + "_wa"], out[key + "_wb"] = wa, wb
        out[key + "_env_auto"] = env_fn(wb, wb, fit)
        out[key + "_env_ab"] = env_fn(wa, wb, fit)
    np.savez_compressed(os.path.join(HERE, "ensemble_ref.npz"), **out)
    print("ensemble_ref.npz written")


def _load_reference_readers():
    """The reference's readers package without its __init__ (which imports camera
    SDKs absent here) and with the LZ4 binding stubbed (only the IM7 path uses it)."""
    import importlib.util
    import types

    R = os.path.join(REF_ROOT, "pivtools_core/image_handling/readers")
    for name, path in (("pivtools_core", os.path.join(REF_ROOT, "pivtools_core")),
                       ("pivtools_core.image_handling", os.path.join(REF_ROOT, "pivtools_core/image_handling")),
                       ("pivtools_core.image_handling.readers", R)):
        m = types.ModuleType(name)
        m.__path__ = [path]
        sys.modules[name] = m
    lz4 = types.ModuleType("lz4")
    lz4b = types.ModuleType("lz4.block")
    lz4.block = lz4b
    sys.modules.setdefault("lz4", lz4)
    sys.modules.setdefault("lz4.block", lz4b)
    spec = importlib.util.spec_from_file_location("pivtools_core.image_handling.readers.pivraw_reader",
                                                  os.path.join(R, "pivraw_reader.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def _pack_mono12p(pix):
    p = pix.reshape(-1, 2).astype(np.uint16)
    b = np.empty((p.shape[0], 3), np.uint8)
    b[:, 0] = p[:, 0] & 0xFF
    b[:, 1] = ((p[:, 0] >> 8) & 0x0F) | ((p[:, 1] & 0x0F) << 4)
    b[:, 2] = p[:, 1] >> 4
    return b.ravel()


def make_ingest():
    """Fixtures for the payload decode of PIVTOOLs Acquisition containers, from
    the reference's own _decode_into (pivraw_reader.py:938-960, which uses
    set_reader.decode_mono12p), driven with minimal header objects over
    temporary container files."""
    import tempfile
    from pathlib import Path
    from types import SimpleNamespace

    pr = _load_reference_readers()
    rng = np.random.default_rng(21)
    W, H, n = 20, 12, 4
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for fmt in ("Mono12p", "BayerRG8"):
            if fmt == "Mono12p":
                frames = rng.integers(0, 4096, (n, H, W))
                dark = rng.integers(0, 300, (2, H, W))
                pay = [_pack_mono12p(f) for f in frames]
                dpay = [_pack_mono12p(d) for d in dark]
            else:
                frames = rng.integers(0, 256, (n, H, W))
                dark = rng.integers(0, 40, (2, H, W))
                pay = [f.astype(np.uint8).ravel() for f in frames]
                dpay = [d.astype(np.uint8).ravel() for d in dark]
            nbytes = pay[0].size
            stride = -(-nbytes // 4096) * 4096
            blob = np.zeros(n * stride, np.uint8)
            dblob = np.zeros(2 * stride, np.uint8)
            for k in range(n):
                blob[k * stride:k * stride + nbytes] = pay[k]
            for k in range(2):
                dblob[k * stride:k * stride + nbytes] = dpay[k]
            fpath = Path(tmp) / f"Camera1_{fmt}.pivraw"
            dpath = Path(tmp) / f"dark_{fmt}.pivraw"
            blob.tofile(fpath)
            dblob.tofile(dpath)
            for q in (fpath, dpath):
                for ext in (".json", ".idx"):
                    Path(str(q) + ext).write_text("{}")
            shape = (H // 2, W // 2) if fmt == "BayerRG8" else (H, W)
            hdr = SimpleNamespace(path=fpath, frame_stride=stride, bytes_per_frame=nbytes, pixel_format=fmt,
                                  width=W, height=H, image_shape=shape, n_frames=n, mode="double_frame")
            dhdr = SimpleNamespace(path=dpath, frame_stride=stride, bytes_per_frame=nbytes, pixel_format=fmt,
                                   width=W, height=H, image_shape=shape, n_frames=2, mode="double_frame")
            out[f"{fmt}_raw"] = blob
            out[f"{fmt}_dark"] = dblob
            out[f"{fmt}_stride"] = np.array(stride)
            for view, k in pr.VIEW_ROTATIONS.items():
                for with_dark in (0, 1):
                    cam = SimpleNamespace(header=hdr, dark=dhdr if with_dark else None, view_rotation=view)
                    oshape = (shape[1], shape[0]) if k % 2 else shape
                    res = np.stack([np.empty(oshape, np.float32) for _ in range(n)])
                    for idx in range(1, n + 1):
                        pr._decode_into(cam, idx, res[idx - 1])
                    out[f"{fmt}_{view}_{with_dark}"] = res
    out["W"], out["H"], out["n"] = np.array(W), np.array(H), np.array(n)
    np.savez_compressed(os.path.join(HERE, "ingest_ref.npz"), **out)
    print("ingest_ref.npz written")


def make_validate():
    """Fixtures for the inter-pass outlier tests from the reference's own
    median_outlier_detection and peak_magnitude_detection
    (pivtools_cli/piv/piv_backend/outlier_detection.py:62-243); its NaN-aware
    median binding (bottleneck, absent here) is given NumPy's nanmedian, the
    same statistic."""
    import importlib.util
    import types

    bn = types.ModuleType("bottleneck")
    bn.nanmedian = np.nanmedian
    sys.modules.setdefault("bottleneck", bn)
    path = os.path.join(REF_ROOT, "pivtools_cli/piv/piv_backend/outlier_detection.py")
    spec = importlib.util.spec_from_file_location("ref_outlier_detection", path)
    od = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(od)
    rng = np.random.default_rng(17)
    out = {}
    for case in range(4):
        ny, nx = 19, 27
        ux = rng.normal(3.0, 0.3, (ny, nx)).astype(np.float32)
        uy = rng.normal(-1.0, 0.3, (ny, nx)).astype(np.float32)
        fail = rng.random((ny, nx)) < 0.04            # failed vectors, zeroed as the driver does
        ux[fail] = 0.0
        uy[fail] = 0.0
        out_idx = rng.integers(0, ny * nx, 6)
        ux.ravel()[out_idx] += rng.normal(0, 4, 6).astype(np.float32)
        masked = np.zeros((ny, nx), bool)
        if case >= 2:
            masked[:, :3] = True
            masked[8:11, 10:14] = True
            ux[masked] = 0.0
            uy[masked] = 0.0
        pk = rng.uniform(0.05, 0.9, (ny, nx)).astype(np.float32)
        for size in (3, 5):
            out[f"c{case}_s{size}_median"] = od.median_outlier_detection(ux, uy, 0.1, 2.0, size,
                                                                         masked=masked if case >= 2 else None)
        out[f"c{case}_ux"], out[f"c{case}_uy"], out[f"c{case}_masked"], out[f"c{case}_pk"] = ux, uy, masked, pk
        out[f"c{case}_peakmag"] = od.peak_magnitude_detection(pk, 0.25)
    np.savez_compressed(os.path.join(HERE, "validate_ref.npz"), **out)
    print("validate_ref.npz written")


def make_infill():
    """Outputs of the reference's infill_harmonic, infill_biharmonic and
    infill_nearest (pivtools_cli/piv/piv_backend/infilling.py:290-421) on
    infill_cases().  The
    module's config import is given the one constant it reads."""
    import importlib.util
    import types

    cfg = types.ModuleType("pivtools_core.config")
    cfg.PREDICTOR_FILL_METHODS = ("harmonic", "nearest", "none")
    pc = types.ModuleType("pivtools_core")
    pc.config = cfg
    sys.modules.setdefault("pivtools_core", pc)
    sys.modules.setdefault("pivtools_core.config", cfg)
    path = os.path.join(REF_ROOT, "pivtools_cli/piv/piv_backend/infilling.py")
    spec = importlib.util.spec_from_file_location("ref_infilling", path)
    inf = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(inf)
    from infill_cases import infill_cases

    out = {}
    for k, c in enumerate(infill_cases()):
        U, V = c["ux"].copy(), c["uy"].copy()
        U[c["fill"]] = np.nan
        V[c["fill"]] = np.nan
        for name, fn in (("harmonic", inf.infill_harmonic), ("biharmonic", inf.infill_biharmonic),
                         ("nearest", inf.infill_nearest)):
            fu, fv = fn(U, V, c["fill"], spacing=c["pitch"], exclude=c["exclude"])
            out[f"c{k}_{name}_ux"] = np.asarray(fu, np.float64)
            out[f"c{k}_{name}_uy"] = np.asarray(fv, np.float64)
    np.savez_compressed(os.path.join(HERE, "infill_ref.npz"), **out)
    print("infill_ref.npz written")


def results_inputs():
    """Seeded per-pass fields of one pair over three passes (NaNs, masked windows,
    values beyond the float16 range, every reason code)."""
    rng = np.random.default_rng(23)
    out = {}
    for k, (ny, nx, win) in enumerate(((3, 4, 16), (4, 5, 8), (6, 7, 8))):
        pre = f"p{k}_"
        ux = rng.normal(2.0, 1.0, (ny, nx)).astype(np.float32)
        uy = rng.normal(-1.0, 1.0, (ny, nx)).astype(np.float32)
        ux[0, 0] = 7.0e4
        uy[-1, -1] = -9.0e4
        b_mask = np.zeros((ny, nx), bool)
        b_mask[0, 1] = True
        reason = rng.choice(np.array([0, 0, 0, 1, 6, 9, 10, 12, 13], np.int8), (ny, nx)).astype(np.int8)
        reason[b_mask] = -1
        nan_mask = reason != 0
        ux[b_mask] = 0.0
        uy[b_mask] = 0.0
        pk_h = rng.uniform(0.0, 2.0, (1, ny, nx)).astype(np.float32)
        pk_h[0][reason == 6] = np.nan
        out.update({
            pre + "ux": ux, pre + "uy": uy, pre + "b_mask": b_mask, pre + "nan_mask": nan_mask,
            pre + "nan_reason": reason, pre + "peak_mag": pk_h,
            pre + "peak_ratio": rng.uniform(1.0, 1.0e5, (ny, nx)).astype(np.float32),
            pre + "peak_choice": np.where(nan_mask, 0, 1).astype(np.intp),
            pre + "predictor": rng.normal(0, 3, (ny, nx, 2)).astype(np.float32),
            pre + "win_ctrs_x": np.linspace(8, 8 + 16 * (nx - 1), nx, dtype=np.float32),
            pre + "win_ctrs_y": np.linspace(8, 8 + 16 * (ny - 1), ny, dtype=np.float32),
            pre + "window_size": np.array([win, win]),
            pre + "planes": rng.normal(0, 1, (ny, nx, win, win)).astype(np.float32),
            pre + "pk_loc_x_raw": rng.normal(0, 1, (1, ny, nx)).astype(np.float32),
            pre + "pk_loc_y_raw": rng.normal(0, 1, (1, ny, nx)).astype(np.float32),
            pre + "sx": rng.uniform(1, 2, (1, ny, nx)).astype(np.float32),
            pre + "sy": rng.uniform(1, 2, (1, ny, nx)).astype(np.float32),
            pre + "sxy": rng.normal(0, 0.1, (1, ny, nx)).astype(np.float32),
        })
    return out


def make_results():
    """Result files written by the reference's own writers
    (pivtools_cli/piv/save_results.py:23-172) from seeded per-pass fields:
    B00007.mat (full), B00008.mat (minimal, passes 1-2 only), B00007's
    correlation-plane npz.  The inputs go to results_in.npz."""
    import shutil

    sys.path.insert(0, REF_ROOT)
    from pivtools_cli.piv import save_results as sr
    from pivtools_cli.piv.piv_result import PIVPassResult, PIVResult

    d = results_inputs()
    res = PIVResult()
    for k in range(3):
        g = lambda key: d[f"p{k}_{key}"]
        ny, nx = g("ux").shape
        res.add_pass(PIVPassResult(
            n_windows=np.array([ny, nx], dtype=np.int32), ux_mat=g("ux"), uy_mat=g("uy"), nan_mask=g("nan_mask"),
            nan_reason=g("nan_reason"), peak_mag=g("peak_mag"), peak_ratio=g("peak_ratio"),
            peak_choice=g("peak_choice"), predictor_field=g("predictor"), b_mask=g("b_mask"),
            window_size=[int(v) for v in g("window_size")], win_ctrs_x=g("win_ctrs_x"),
            win_ctrs_y=g("win_ctrs_y"),
            debug_dump={"planes": g("planes"), "peak_finder": 3, "pk_loc_x_raw": g("pk_loc_x_raw"),
                        "pk_loc_y_raw": g("pk_loc_y_raw"), "pk_height_raw": g("peak_mag"),
                        "pk_ratio_raw": g("peak_ratio"), "sx": g("sx"), "sy": g("sy"), "sxy": g("sxy")}))
    out = os.path.join(HERE, "results_ref")
    if os.path.isdir(out):
        shutil.rmtree(out)
    sr.save_piv_result_distributed(res, out, 7)
    sr.save_piv_result_distributed(res, out, 8, runs_to_save=[1, 2], save_mode="minimal")
    dump = sr.save_corr_plane_dump(res, out, 7)
    # keep the arrays; of the two text entries keep only the label codes
    z = dict(np.load(dump))
    codes = sorted(int(c) for c in __import__("json").loads(str(z.pop("nan_reason_labels"))))
    z.pop("pk_origin_note")
    z["nan_reason_label_codes"] = np.array(codes, np.int64)
    np.savez_compressed(dump, **z)
    np.savez_compressed(os.path.join(HERE, "results_in.npz"), **d)
    print("results_ref/ and results_in.npz written")


def make_floor():
    """Coloured-floor P grids and the per-window lookup from the reference's own
    build_P_grid / interp_P (pivtools_cli/piv/piv_backend/kspace_floor_psd.py:206-275)
    on 16 x 16 windows, with the fractions the ensemble driver derives from a
    float32 predictor (single_pass_accumulator.py:852-853)."""
    sys.path.insert(0, REF_ROOT)
    sys.path.insert(0, os.path.join(ROOT, "python-pivtools_b200"))
    from pivtools_cli.piv.piv_backend import kspace_floor_psd as K
    from pivtools_cli.piv.piv_backend.interpolation_noise_psd import frac_distance
    from pivtools_b200 import geometry
    from pivtools_b200.ensemble import pair_envelope

    rng = np.random.default_rng(31)
    out = {}
    cases = [("lanczos", True, "square"), ("lanczos", False, "gaussian"), ("cubic", True, "gaussian"),
             ("cubic", False, "square")]
    for ci, (kernel, hole, wt) in enumerate(cases):
        w = geometry.window_weight((16, 16), wt).astype(np.float32)
        env = pair_envelope(w, w, (16, 16)) if wt == "gaussian" else np.ones((16, 16))
        fs, P = K.build_P_grid(env, kernel, hole, w, n_fracs=5)
        out[f"c{ci}_w"], out[f"c{ci}_env"], out[f"c{ci}_fs"], out[f"c{ci}_P"] = w, env, fs, P
    pdy = rng.normal(0.0, 3.0, 64).astype(np.float32)
    pdx = rng.normal(0.0, 3.0, 64).astype(np.float32)
    pdx[:8] = np.array([0.0, 1.0, -1.0, 0.5, -0.5, 0.25, 2.0, 3.0], np.float32)   # nodes and half steps
    fx, fy = frac_distance(pdx / 2.0), frac_distance(pdy / 2.0)
    out["pred_dy"], out["pred_dx"] = pdy, pdx
    for ci in range(len(cases)):
        out[f"c{ci}_Pwin"] = K.interp_P(out[f"c{ci}_fs"], out[f"c{ci}_P"], fx, fy).astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "floor_ref.npz"), **out)
    print("floor_ref.npz written")


def make_vmask():
    """Per-pass vector masks from the reference's own compute_vector_mask
    (pivtools_core/image_handling/load_images.py:827-990), compiled on its own
    with the reference's window_utils; its image-shape guard is skipped (the
    fixture masks have the image shape)."""
    import logging
    from types import SimpleNamespace

    sys.path.insert(0, REF_ROOT)
    from pivtools_core import window_utils as wu

    (cvm,) = _reference_functions(os.path.join(REF_ROOT, "pivtools_core/image_handling/load_images.py"),
                                  ["compute_vector_mask"])
    cvm.__globals__.update(logging=logging, compute_window_centers=wu.compute_window_centers,
                           compute_window_centers_single_mode=wu.compute_window_centers_single_mode,
                           require_mask_fits_camera=lambda *a, **k: None, List=list)
    rng = np.random.default_rng(41)
    out = {}
    ws, ov = [(64, 64), (32, 32), (16, 16)], [50, 50, 75]
    for ci, (H, W) in enumerate(((512, 384), (300, 257))):
        pm = np.zeros((H, W), bool)
        pm[100:180, 50:200] = True
        yy, xx = np.mgrid[:H, :W]
        pm |= (yy - 0.6 * H) ** 2 + (xx - 0.3 * W) ** 2 < 40 ** 2
        pm[rng.random((H, W)) < 0.02] = True
        out[f"c{ci}_pixel_mask"] = pm
        for ti, thr in enumerate((0.0, 0.5, 0.9)):
            cfg = SimpleNamespace(image_shape_for=lambda cam, H=H, W=W: (H, W), mask_threshold=thr, num_passes=3,
                                  window_sizes=ws, overlap=ov, ensemble_piv=False)
            for k, vm in enumerate(cvm(pm, cfg, 1, ensemble=False)):
                out[f"c{ci}_t{ti}_p{k}"] = vm
    np.savez_compressed(os.path.join(HERE, "vmask_ref.npz"), **out)
    print("vmask_ref.npz written")


def make_xcorr():
    """Outputs of the reference's compiled bulkxcorr2d and
    bulkxcorr2d_accumulate_triple on the seeded cases of xcorr_cases.py."""
    import xcorr_cases as XC

    if O.ref_bulk() is None:
        raise SystemExit("build the reference correlator first: make -C oracle ref")
    out = {}
    names = []
    for c in XC.all_cases():
        r = O.ref_bulkxcorr2d(c["A"], c["B"], c["mask"], c["cx"], c["cy"], c["win"], c["wa"], c["wb"],
                              n_peaks=c["n_peaks"], peak_finder=c["finder"], ensemble=c["ensemble"],
                              want_planes=len(c["plane_idx"]) > 0, peakfit_impl=c["impl"])
        nm = c["name"]
        names.append(nm)
        out[f"{nm}__error"] = np.int32(r["error"])
        out[f"{nm}__checksum"] = np.float64(XC.checksum(c))
        for k in XC.OUT_KEYS:
            out[f"{nm}__{k}"] = r[k]
        if len(c["plane_idx"]):
            h, w = c["win"]
            out[f"{nm}__planes"] = r["planes"].reshape(-1, h, w)[c["plane_idx"]]
    out["names"] = np.array(names)
    # loss-of-correlation weight numel / (wB (*) wB) as bulkxcorr2d forms it
    # (PIV_2d_cross_correlate.c:216-222 over xcorr.c's convolve)
    L = O.ref_bulk()
    L.convolve.argtypes = [O._f32, O._f32, O._f32, O._i32]
    L.convolve.restype = ctypes.c_uint
    from pivtools_b200 import geometry

    cw_sizes = sorted({c["win"] for c in XC.all_cases()})
    for (h, w) in cw_sizes:
        for wt in ("gaussian", "blackman", "square"):
            wb = geometry.window_weight((h, w), wt).ravel()
            conv = np.zeros(h * w, np.float32)
            assert L.convolve(wb, wb, conv, np.array([h, w], np.int32)) == 0
            out[f"cw_{wt}_{h}x{w}"] = (np.float32(h * w) / conv).reshape(h, w)
    out["cw_sizes"] = np.array(cw_sizes, np.int32)
    np.savez_compressed(os.path.join(HERE, "xcorr_ref.npz"), **out)
    print("xcorr_ref.npz written:", len(names), "cases")
    tout = {}
    tnames = []
    for c in XC.triple_cases():
        s = O.ref_accumulate_triple(c["A"], c["B"], np.zeros((len(c["cy"]), len(c["cx"])), np.float32),
                                    c["cx"], c["cy"], c["win"], *c["w"], fit_size=c["fit"],
                                    mean_subtract=c["ms"], per_pair_norm=c["pn"])
        tnames.append(c["name"])
        for k, v in zip(("ab", "aa", "bb"), s):
            tout[f"{c['name']}__{k}"] = v.reshape(-1, *v.shape[2:])[c["keep"]]
    tout["names"] = np.array(tnames)
    np.savez_compressed(os.path.join(HERE, "triple_ref.npz"), **tout)
    print("triple_ref.npz written:", len(tnames), "cases")


def _load_reference_module(name):
    """One module of the reference's readers package (the package stubs of
    _load_reference_readers already in place), the LZ4 binding standing in for
    python-lz4 where that is absent."""
    import importlib.util

    import lavision_oracle as LO

    LO.install_lz4_stub()
    _load_reference_readers()
    R = os.path.join(REF_ROOT, "pivtools_core/image_handling/readers")
    full = "pivtools_core.image_handling.readers." + name
    if full in sys.modules and getattr(sys.modules[full], "__file__", None):
        return sys.modules[full]
    spec = importlib.util.spec_from_file_location(full, os.path.join(R, name + ".py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[full] = mod
    spec.loader.exec_module(mod)
    return mod


def _frames_u16(rng, F, H, W):
    """Camera-like uint16 frames: a smooth background, particles and noise, so the
    token coder meets small deltas (nibble runs, int8) and large jumps alike."""
    yy, xx = np.mgrid[0:H, 0:W]
    out = np.empty((F, 1, H, W), np.uint16)
    for k in range(F):
        img = 500 + 40 * np.sin(xx / 7.0 + k) + 30 * np.cos(yy / 5.0)
        img += rng.integers(0, 4, (H, W))
        for _ in range(max(1, H * W // 40)):
            y, x = rng.integers(0, H), rng.integers(0, W)
            img[y, x] += rng.integers(200, 4000)
        out[k, 0] = np.clip(img, 0, 65535).astype(np.uint16)
    return out


def make_pfill():
    """Outputs of the reference's fill_masked_predictor with method 'nearest'
    (pivtools_cli/piv/piv_backend/infilling.py:808-874, 114-141: the nearest
    unmasked node in physical distance, scipy's Euclidean distance transform
    choosing among equidistant donors) on seeded (N, ny, nx, 2) predictor fields
    with blob, edge and stripe masks and isotropic and anisotropic pitches."""
    import importlib.util
    import types

    cfg = types.ModuleType("pivtools_core.config")
    cfg.PREDICTOR_FILL_METHODS = ("harmonic", "nearest", "none")
    pc = types.ModuleType("pivtools_core")
    pc.config = cfg
    sys.modules.setdefault("pivtools_core", pc)
    sys.modules.setdefault("pivtools_core.config", cfg)
    path = os.path.join(REF_ROOT, "pivtools_cli/piv/piv_backend/infilling.py")
    spec = importlib.util.spec_from_file_location("ref_infilling", path)
    inf = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(inf)
    rng = np.random.default_rng(515)
    out = {}
    cases = []
    for k, (ny, nx, pitch) in enumerate([(31, 31, (16.0, 16.0)), (40, 57, (16.0, 8.0)), (25, 64, (12.0, 12.0)),
                                         (63, 63, (32.0, 16.0))]):
        yy, xx = np.mgrid[0:ny, 0:nx]
        m = (yy - ny * 0.45) ** 2 + (xx - nx * 0.6) ** 2 < (min(ny, nx) * 0.22) ** 2
        if k % 2:
            m |= xx < 2                                 # a masked edge
        if k == 2:
            m |= (yy % 7 == 3) & (xx > nx // 3)        # stripes: many equidistant donors
        field = rng.normal(0, 2, (2, ny, nx, 2)).astype(np.float32)
        field[:, m] = 0.0
        filled = inf.fill_masked_predictor(field, m, pitch, "nearest")
        out[f"c{k}_field"] = field
        out[f"c{k}_mask"] = m
        out[f"c{k}_pitch"] = np.array(pitch)
        out[f"c{k}_filled"] = np.asarray(filled, np.float32)
        cases.append(k)
    out["n_cases"] = np.array(len(cases))
    np.savez_compressed(os.path.join(HERE, "pfill_ref.npz"), **out)
    print("pfill_ref.npz written")


def make_outliers():
    """Outputs of the reference's sigma_outlier_detection and div_vort_outliers
    (pivtools_cli/piv/piv_backend/outlier_detection.py:246-381) on seeded fields
    with outliers, zeros and NaN holes (fixture outliers_ref.npz).  The module's
    median binding (bottleneck, absent here; unused by these two tests) is given
    NumPy's nanmedian."""
    import importlib.util
    import types

    bn = types.ModuleType("bottleneck")
    bn.nanmedian = np.nanmedian
    sys.modules.setdefault("bottleneck", bn)

    path = os.path.join(REF_ROOT, "pivtools_cli/piv/piv_backend/outlier_detection.py")
    spec = importlib.util.spec_from_file_location("ref_outliers", path)
    od = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(od)
    rng = np.random.default_rng(616)
    out = {}
    for k, (ny, nx) in enumerate([(31, 31), (40, 57), (63, 63), (9, 12)]):
        yy, xx = np.mgrid[0:ny, 0:nx]
        ux = (2.0 + np.sin(xx / 5.0) + 0.1 * rng.normal(size=(ny, nx))).astype(np.float32)
        uy = (-1.0 + np.cos(yy / 4.0) + 0.1 * rng.normal(size=(ny, nx))).astype(np.float32)
        bad = rng.random((ny, nx)) < 0.05
        ux[bad] += rng.uniform(-8, 8, bad.sum()).astype(np.float32)
        uy[bad] += rng.uniform(-8, 8, bad.sum()).astype(np.float32)
        if k % 2:
            holes = rng.random((ny, nx)) < 0.04
            ux[holes] = np.nan
            uy[holes] = np.nan
        zero = rng.random((ny, nx)) < 0.03
        ux[zero] = 0.0
        uy[zero] = 0.0
        out[f"c{k}_ux"], out[f"c{k}_uy"] = ux, uy
        for thr in (1.5, 2.0, 3.0):
            out[f"c{k}_sigma_{thr}"] = od.sigma_outlier_detection(ux, uy, sigma_threshold=thr)
        out[f"c{k}_divvort"] = od.div_vort_outliers(ux, uy)
        out[f"c{k}_divvort_given"] = od.div_vort_outliers(ux, uy, div_thresh=0.5, vort_thresh=0.7)
    out["n_cases"] = np.array(4)
    np.savez_compressed(os.path.join(HERE, "outliers_ref.npz"), **out)
    print("outliers_ref.npz written")


def make_lavision():
    """Fixtures of the LaVision decode: .im7 files of every pack type (written by
    oracle/lavision_oracle.py) with the reference reader's read_im7 and
    read_im7_camera results; the reference's own lvpyio fixtures (pack 1 and
    version-1 pack 20, decoded by LaVision's lvpyio 1.3.1); .set entry payloads
    under every codec and decoder with the reference's _decompress_entry and
    _decode_pixels results."""
    import json
    import tempfile
    import types
    import zlib

    import lavision_oracle as LO

    im7 = _load_reference_module("im7_reader")
    st = _load_reference_module("set_reader")
    rng = np.random.default_rng(2024)
    out, meta = {}, {"im7": [], "lvpyio": [], "set": []}

    def attrs(slope, offset):
        return LO.im7_attributes(slope, offset)

    cases = []
    fr = _frames_u16(rng, 3, 20, 24)
    cases.append(("p0_word", LO.im7_pack0(fr, attrs(2.5, 100.0)), [(2, 1, None), (1, 2, 1)]))
    ff = rng.normal(0, 50, (2, 1, 12, 16)).astype(np.float32)
    cases.append(("p0_float", LO.im7_pack0(ff, attrs(None, None)), [(1, 2, None)]))
    fr1 = _frames_u16(rng, 3, 18, 22)
    cases.append(("p1_tokens", LO.im7_pack1(fr1, attrs(0.5, None), rng), [(2, 1, None), (1, 2, None), (3, 1, None)]))
    fr1b = _frames_u16(rng, 1, 40, 33)
    cases.append(("p1_single", LO.im7_pack1(fr1b, attrs(None, None), rng), [(1, 2, None)]))
    fr2 = _frames_u16(rng, 2, 16, 20)
    cases.append(("p2_rows", LO.im7_pack2(fr2, attrs(1.0, -3.0), per_row=True), [(2, 1, None), (1, 2, None)]))
    fr2b = _frames_u16(rng, 1, 16, 20)
    cases.append(("p2_frame", LO.im7_pack2(fr2b, attrs(None, None), per_row=False), [(1, 1, None)]))
    fr20 = _frames_u16(rng, 2, 32, 48)
    cases.append(("p20_v0", LO.im7_pack20_v0(fr20, attrs(3.0, 1.5)), [(1, 2, None), (2, 1, None)]))
    fr20b = _frames_u16(rng, 4, 24, 40)
    cases.append(("p20_v1", LO.im7_pack20_v1(fr20b, attrs(None, None)), [(1, 2, None), (2, 2, 1)]))
    with tempfile.TemporaryDirectory() as td:
        for name, blob, cams in cases:
            path = os.path.join(td, name + ".im7")
            with open(path, "wb") as f:
                f.write(blob)
            _, px, sc = im7.read_im7(path)
            out[name + "_file"] = np.frombuffer(blob, np.uint8)
            out[name + "_pixels"] = px
            entry = {"name": name, "slope": sc.slope, "offset": sc.offset, "cams": []}
            for i, (cam, fpc, nfr) in enumerate(cams):
                r = im7.read_im7_camera(path, camera_no=cam, frames_per_camera=fpc, frames=nfr)
                out[f"{name}_cam{i}"] = r
                entry["cams"].append([cam, fpc, nfr])
            meta["im7"].append(entry)
    fx = os.path.join(REF_ROOT, "unit-tests", "fixtures")
    for sub, name in (("im7_pack1", "carry_3frames"), ("im7_pack1", "high_nibble_8"),
                      ("im7_v1_pack20", "three_frames")):
        path = os.path.join(fx, sub, name + ".im7")
        with open(path, "rb") as f:
            out[f"lv_{name}_file"] = np.frombuffer(f.read(), np.uint8)
        out[f"lv_{name}_lvpyio"] = np.load(os.path.join(fx, sub, name + ".lvpyio.npy"))
        _, px, _ = im7.read_im7(path)
        out[f"lv_{name}_ref"] = px
        meta["lvpyio"].append(name)
    W, H = 16, 12
    for dec in ("raw-16-bit", "raw-8-bit", "mono-12p", "mono-12pmsb", "mono-12packed", "mono-10p", "mono-10pmsb"):
        nbytes = st._payload_bytes(dec, W, H)
        payload = rng.integers(0, 256, nbytes).astype(np.uint8).tobytes()
        out[f"set_{dec}_pixels"] = st._decode_pixels(payload, dec, W, H)
        out[f"set_{dec}_payload"] = np.frombuffer(payload, np.uint8)
        for codec in ("", "Zlib", "LZ4", "IMX"):
            if codec == "Zlib":
                stored = zlib.compress(payload)
            elif codec == "LZ4":
                stored = LO.lz4_encode(payload)
            elif codec == "IMX":
                stored, _ = LO.tokens_encode(np.frombuffer(payload, "<u2"), 0, rng)
            else:
                stored = payload
            fi = types.SimpleNamespace(codec=codec, frame_idx=0,
                                       data_path=type("P", (), {"name": "x-1.ims",
                                                                "parent": type("Q", (), {"name": "rec"})()})())
            got = st._decompress_entry(stored, fi, 0, nbytes)
            got = bytes(got) if not isinstance(got, np.ndarray) else got.tobytes()
            assert got == payload, (dec, codec)
            out[f"set_{dec}_{codec or 'none'}_stored"] = np.frombuffer(stored, np.uint8)
        meta["set"].append({"decoder": dec, "width": W, "height": H})
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "lavision_ref.npz"), **out)
    print("lavision_ref.npz written")


if __name__ == "__main__":
    what = sys.argv[1:] or ["peakfit", "warp"]
    if "xcorr" in what:
        make_xcorr()
    if "peakfit" in what:
        make_peakfit()
    if "warp" in what:
        make_warp()
    if "kspace" in what:
        make_kspace()
    if "kspace_c" in what:
        make_kspace_c()
    if "ensemble" in what:
        make_ensemble()
    if "ingest" in what:
        make_ingest()
    if "validate" in what:
        make_validate()
    if "results" in what:
        make_results()
    if "floor" in what:
        make_floor()
    if "vmask" in what:
        make_vmask()
    if "infill" in what:
        make_infill()
    if "lavision" in what:
        make_lavision()
    if "pfill" in what:
        make_pfill()
    if "outliers" in what:
        make_outliers()
