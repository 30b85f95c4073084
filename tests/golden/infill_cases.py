"""Seeded inputs of the infill fixture (infill_ref.npz, made by
`make_golden.py infill` from the reference's infill_harmonic / infill_biharmonic);
the tests rebuild them here."""

import numpy as np


def infill_cases():
    """Seeded fields and fill masks of the infill fixture: smooth fields with
    scattered holes, a clustered hole, holes on the frame edge and corner,
    anisotropic pitch, and an excluded (masked) block."""
    rng = np.random.default_rng(23)
    cases = []
    for k, (ny, nx, pitch) in enumerate(((23, 31, (16.0, 16.0)), (40, 28, (8.0, 16.0)), (63, 63, (16.0, 16.0)))):
        yy, xx = np.mgrid[0:ny, 0:nx]
        ux = (3.0 + np.sin(xx / 6.0) + yy / 9.0 + 0.05 * rng.normal(size=(ny, nx))).astype(np.float32)
        uy = (-1.0 + np.cos(yy / 5.0) - xx / 11.0 + 0.05 * rng.normal(size=(ny, nx))).astype(np.float32)
        fill = rng.random((ny, nx)) < 0.06
        fill[5:9, 7:12] = True                 # a cluster
        fill[0, 0:3] = True                    # frame corner and edge
        fill[ny - 1, nx // 2] = True
        excl = np.zeros((ny, nx), bool)
        if k >= 1:
            excl[12:16, 2:6] = True            # masked windows: neither filled nor donors
            fill &= ~excl
            ux[excl] = 0.0
            uy[excl] = 0.0
        cases.append(dict(ux=ux, uy=uy, fill=fill, exclude=excl if k >= 1 else None, pitch=pitch))
    return cases
