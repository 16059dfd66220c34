"""ORACLE (test infrastructure): the arithmetic of the reference's save_detected_geotiff
(src/form_image_pfa.py:249-299), restated with NumPy; rasterio and pyproj are replaced by a ``to_map``
callable and by returning the pixels instead of writing them.

* ``display_u8``: amp = |img| as float32, hi = np.percentile(amp, 99.7),
  np.clip(amp / (hi + 1e-12) * 255.0, 0, 255).astype(np.uint8)               (:287-292)
* ``affine``: the rotated radar-grid -> map affine from the scene centre and the per-pixel ground
  displacements, rasterio's Affine(a, b, c, d, e, f) order                   (:268-282)
"""
from __future__ import annotations

import numpy as np


def display_u8(img, percentile=99.7):
    amp = np.abs(img).astype(np.float32)
    hi = np.percentile(amp, percentile)
    return np.clip(amp / (hi + 1e-12) * 255.0, 0, 255).astype(np.uint8), hi


def affine(shape, geo, center_ecef, uiax, uiay, to_map, flip_col=False, flip_row=False):
    m, n = shape
    row0, col0 = m // 2, n // 2
    dhat = np.array(geo["dhat"])
    chat = np.array(geo["chat"])
    sc = -1.0 if flip_col else 1.0
    sr = -1.0 if flip_row else 1.0
    v_col = sc * geo["dr"] * (dhat[0] * uiax + dhat[1] * uiay)
    v_row = sr * geo["dc"] * (chat[0] * uiax + chat[1] * uiay)
    p0, pcol, prow = to_map(center_ecef), to_map(center_ecef + v_col), to_map(center_ecef + v_row)
    a = pcol - p0
    b = prow - p0
    return (a[0], b[0], p0[0] - a[0] * col0 - b[0] * row0, a[1], b[1], p0[1] - a[1] * col0 - b[1] * row0)
