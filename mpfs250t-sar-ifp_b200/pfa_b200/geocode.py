"""Geocoding of the float image: the map affine and display scaling of ``save_detected_geotiff``
(src/form_image_pfa.py:249-299), without rasterio or pyproj.

The reference's image is planar, so one affine maps the radar grid (col = range, row = cross) to UTM: it
projects the scene-centre ECEF point and the centre displaced by one pixel along each grid axis (per-pixel
ground vectors dr (dhat . (uIAX, uIAY)) and dc (chat . (uIAX, uIAY))) and takes differences.  Here the
ECEF -> UTM projection is this module's own FP64 code: geodetic latitude/longitude on WGS84 (iterated to
convergence) and the transverse Mercator projection by the Krueger series to sixth order in the third
flattening (Karney, "Transverse Mercator with an accuracy of a few nanometers", J. Geodesy 85, 2011), the
accuracy class of the projection pyproj applies for UTM.

``display_u8`` runs the reference's 99.7-percentile scaling on the device (``pfa_display_u8``);
``write_geotiff`` writes a single-band GeoTIFF with a ModelTransformationTag (rotated affine) and the
projected CRS key.  The file is uncompressed (the reference asks rasterio for LZW); its pixels, size, CRS
and transform are the reference's.
"""
from __future__ import annotations

import ctypes as C
import math
import struct

import numpy as np

from . import _lib

# WGS84
WGS84_A = 6378137.0
WGS84_F = 1.0 / 298.257223563
UTM_K0 = 0.9996


# ----------------------------------------------------------------------------- geodesy
def geodetic_to_ecef(lon_deg, lat_deg, h=0.0):
    a, f = WGS84_A, WGS84_F
    e2 = f * (2.0 - f)
    lat, lon = math.radians(lat_deg), math.radians(lon_deg)
    nn = a / math.sqrt(1.0 - e2 * math.sin(lat) ** 2)
    return np.array([(nn + h) * math.cos(lat) * math.cos(lon), (nn + h) * math.cos(lat) * math.sin(lon),
                     (nn * (1.0 - e2) + h) * math.sin(lat)])


def ecef_to_geodetic(x, y, z):
    """(lon_deg, lat_deg, h) of an ECEF point on WGS84: fixed-point iteration
    lat <- atan2(z + e^2 N(lat) sin(lat), p), to convergence."""
    a, f = WGS84_A, WGS84_F
    e2 = f * (2.0 - f)
    lon = math.atan2(y, x)
    p = math.hypot(x, y)
    lat = math.atan2(z, p * (1.0 - e2))
    for _ in range(100):
        s = math.sin(lat)
        nn = a / math.sqrt(1.0 - e2 * s * s)
        nxt = math.atan2(z + e2 * nn * s, p)
        done = abs(nxt - lat) < 1e-15
        lat = nxt
        if done:
            break
    s, c = math.sin(lat), math.cos(lat)
    nn = a / math.sqrt(1.0 - e2 * s * s)
    h = p / c - nn if abs(c) > 1e-3 else abs(z) / abs(s) - nn * (1.0 - e2)
    return math.degrees(lon), math.degrees(lat), h


def utm_epsg_auto(center_ecef):
    """The reference's automatic zone: (32600 north / 32700 south) + int((lon + 180) // 6) + 1."""
    lon, lat, _ = ecef_to_geodetic(*center_ecef)
    return (32600 if lat >= 0 else 32700) + int((lon + 180) // 6) + 1


def _krueger():
    n = WGS84_F / (2.0 - WGS84_F)
    n2, n3, n4, n5, n6 = n ** 2, n ** 3, n ** 4, n ** 5, n ** 6
    big_a = WGS84_A / (1.0 + n) * (1.0 + n2 / 4.0 + n4 / 64.0 + n6 / 256.0)
    alpha = (n / 2.0 - 2.0 * n2 / 3.0 + 5.0 * n3 / 16.0 + 41.0 * n4 / 180.0 - 127.0 * n5 / 288.0 + 7891.0 * n6 / 37800.0,
             13.0 * n2 / 48.0 - 3.0 * n3 / 5.0 + 557.0 * n4 / 1440.0 + 281.0 * n5 / 630.0 - 1983433.0 * n6 / 1935360.0,
             61.0 * n3 / 240.0 - 103.0 * n4 / 140.0 + 15061.0 * n5 / 26880.0 + 167603.0 * n6 / 181440.0,
             49561.0 * n4 / 161280.0 - 179.0 * n5 / 168.0 + 6601661.0 * n6 / 7257600.0,
             34729.0 * n5 / 80640.0 - 3418889.0 * n6 / 1995840.0,
             212378941.0 * n6 / 319334400.0)
    return n, big_a, alpha


_N, _A, _ALPHA = _krueger()


def utm_forward(lon_deg, lat_deg, epsg):
    """(easting, northing) in metres of a WGS84 point in the UTM zone of ``epsg`` (326zz north, 327zz south)."""
    zone = epsg % 100
    south = epsg // 100 == 327
    lon0 = math.radians((zone - 1) * 6 - 180 + 3)
    lat = math.radians(lat_deg)
    lam = math.radians(lon_deg) - lon0
    e = 2.0 * math.sqrt(_N) / (1.0 + _N)
    s = math.sin(lat)
    t = math.sinh(math.atanh(s) - e * math.atanh(e * s))
    xi_p = math.atan2(t, math.cos(lam))
    eta_p = math.atanh(math.sin(lam) / math.sqrt(1.0 + t * t))
    xi, eta = xi_p, eta_p
    for j, al in enumerate(_ALPHA, start=1):
        xi += al * math.sin(2 * j * xi_p) * math.cosh(2 * j * eta_p)
        eta += al * math.cos(2 * j * xi_p) * math.sinh(2 * j * eta_p)
    return 500000.0 + UTM_K0 * _A * eta, (10000000.0 if south else 0.0) + UTM_K0 * _A * xi


def ecef_to_utm(p, epsg):
    lon, lat, _ = ecef_to_geodetic(*p)
    return np.array(utm_forward(lon, lat, epsg))


# ----------------------------------------------------------------------------- affine
def geotransform(shape, geo, center_ecef, uiax, uiay, epsg="auto", flip_col=False, flip_row=False, to_map=None):
    """(epsg, (a, b, c, d, e, f)) with x = a col + b row + c, y = d col + e row + f: the rotated affine of
    save_detected_geotiff (src/form_image_pfa.py:262-282) for an image of ``shape`` (rows = cross, cols =
    range, centred).  ``geo`` carries dr, dc, dhat, chat (resample_kspace); ``to_map`` overrides the
    ECEF -> map projection (default: UTM of ``epsg``)."""
    center_ecef = np.asarray(center_ecef, np.float64)
    uiax, uiay = np.asarray(uiax, np.float64), np.asarray(uiay, np.float64)
    if epsg in (None, "auto"):
        epsg = utm_epsg_auto(center_ecef)
    proj = to_map if to_map is not None else (lambda p: ecef_to_utm(p, epsg))
    m, n = shape
    row0, col0 = m // 2, n // 2
    dhat, chat = np.array(geo["dhat"]), np.array(geo["chat"])
    sc = -1.0 if flip_col else 1.0
    sr = -1.0 if flip_row else 1.0
    v_col = sc * geo["dr"] * (dhat[0] * uiax + dhat[1] * uiay)      # ground step of +1 col (range)
    v_row = sr * geo["dc"] * (chat[0] * uiax + chat[1] * uiay)      # ground step of +1 row (cross)
    p0, pcol, prow = proj(center_ecef), proj(center_ecef + v_col), proj(center_ecef + v_row)
    a, b = pcol - p0, prow - p0
    return epsg, (a[0], b[0], p0[0] - a[0] * col0 - b[0] * row0, a[1], b[1], p0[1] - a[1] * col0 - b[1] * row0)


# ----------------------------------------------------------------------------- display scaling
def display_u8(mag, percentile: float = 99.7, stream=None):
    """uint8 display image of a float32 magnitude CUDA tensor (the reference's 99.7-percentile scaling),
    on the device.  Returns (uint8 tensor of mag's shape, hi as a float32 0-d tensor)."""
    import torch
    from .engine import _stream_handle
    lib = _lib.load()
    if mag.dtype != torch.float32 or not mag.is_cuda:
        raise ValueError("mag must be a float32 CUDA tensor")
    mag = mag.contiguous()
    out = torch.empty(mag.shape, dtype=torch.uint8, device=mag.device)
    ws = torch.empty(int(lib.pfa_display_workspace_bytes()), dtype=torch.uint8, device=mag.device)
    hi = torch.empty((), dtype=torch.float32, device=mag.device)
    _lib.check(lib.pfa_display_u8(C.c_void_p(mag.data_ptr()), C.c_int64(mag.numel()), C.c_float(percentile),
                                  C.c_void_p(ws.data_ptr()), C.c_void_p(out.data_ptr()), C.c_void_p(hi.data_ptr()),
                                  _stream_handle(stream)))
    return out, hi


# ----------------------------------------------------------------------------- GeoTIFF
def write_geotiff(path, data, epsg, affine):
    """Single-band baseline GeoTIFF (little endian, uncompressed, strips of 64 rows) of a uint8, uint16 or
    float32 image with ModelTransformationTag = the affine and ProjectedCSTypeGeoKey = epsg."""
    data = np.ascontiguousarray(data)
    fmt = {np.dtype(np.uint8): (8, 1), np.dtype(np.uint16): (16, 1), np.dtype(np.float32): (32, 3)}
    if data.ndim != 2 or data.dtype not in fmt:
        raise ValueError("data must be a 2-D uint8, uint16 or float32 array")
    bits, sfmt = fmt[data.dtype]
    h, w = data.shape
    rps = 64
    nstrips = (h + rps - 1) // rps
    counts = [min(rps, h - k * rps) * w * data.dtype.itemsize for k in range(nstrips)]
    a, b, c, d, e, f = (float(v) for v in affine)
    mtx = (a, b, 0.0, c, d, e, 0.0, f, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0)
    geokeys = (1, 1, 0, 3, 1024, 0, 1, 1, 1025, 0, 1, 1, 3072, 0, 1, int(epsg))
    # (tag, type, values): type 3 SHORT, 4 LONG, 12 DOUBLE; tags ascending; strip offsets filled in below
    entries = [[256, 4, (w,)], [257, 4, (h,)], [258, 3, (bits,)], [259, 3, (1,)], [262, 3, (1,)],
               [273, 4, (0,) * nstrips], [277, 3, (1,)], [278, 4, (rps,)], [279, 4, tuple(counts)], [284, 3, (1,)],
               [339, 3, (sfmt,)], [34264, 12, mtx], [34735, 3, geokeys]]
    size = {3: 2, 4: 4, 12: 8}
    code = {3: "H", 4: "I", 12: "d"}
    pos = 8 + 2 + 12 * len(entries) + 4                  # header, IFD; then the out-of-line values
    where = {}
    for tag, typ, vals in entries:
        nbytes = len(vals) * size[typ]
        if nbytes > 4:
            pos += pos & 7 and 8 - (pos & 7)               # 8-byte aligned (doubles)
            where[tag] = pos
            pos += nbytes
    data_off = pos + (pos & 7 and 8 - (pos & 7))
    entries[5][2] = tuple(data_off + sum(counts[:k]) for k in range(nstrips))
    out = bytearray(b"II*\x00" + struct.pack("<I", 8) + struct.pack("<H", len(entries)))
    blobs = []
    for tag, typ, vals in entries:
        raw = struct.pack("<" + code[typ] * len(vals), *vals)
        if tag in where:
            out += struct.pack("<HHII", tag, typ, len(vals), where[tag])
            blobs.append((where[tag], raw))
        else:
            out += struct.pack("<HHI", tag, typ, len(vals)) + raw.ljust(4, b"\x00")
    out += struct.pack("<I", 0)                            # no next IFD
    for off, raw in blobs:
        out += b"\x00" * (off - len(out)) + raw
    out += b"\x00" * (data_off - len(out))
    out += data.astype(data.dtype.newbyteorder("<"), copy=False).tobytes()
    with open(path, "wb") as fh:
        fh.write(out)
    return path


def save_detected_geotiff(mag, tables, out_tif, epsg="auto", flip_col=False, flip_row=False, dtype="uint8",
                          stream=None):
    """Drop-in for save_detected_geotiff (src/form_image_pfa.py:249-299) on the engine's detected image:
    ``mag`` is the float32 |img| (m2, n2) CUDA tensor of FloatPlan.form (centred layout), ``tables`` the
    prepare_tables dict (geo, center_ecef, uiax, uiay).  dtype "uint8" (the reference's default, scaled on
    the device) or "float32" (raw magnitude).  Returns (path, epsg, affine)."""
    epsg, aff = geotransform(tuple(mag.shape), tables["geo"], tables["center_ecef"], tables["uiax"], tables["uiay"],
                             epsg, flip_col, flip_row)
    if dtype == "float32":
        data = mag.float().cpu().numpy()
    elif dtype == "uint8":
        data = display_u8(mag, 99.7, stream)[0].cpu().numpy()
    else:
        raise ValueError("dtype must be 'uint8' or 'float32'")
    write_geotiff(out_tif, data, epsg, aff)
    return out_tif, epsg, aff
