"""CPU: the geocoding half of save_detected_geotiff (src/form_image_pfa.py:249-299) without pyproj or
rasterio: WGS84 geodesy, the UTM projection (checked against properties that define it: the central
meridian's false easting and scaled meridian arc, integrated numerically here, conformality, the southern
false northing), the reference's zone rule, the rotated affine against the restated reference arithmetic,
and the GeoTIFF file read back by PIL."""
import math

import numpy as np
import pytest

from oracle import geotiff_ref
from pfa_b200 import geocode as gc


@pytest.mark.parametrize("lon,lat,h", [(-96.8, 46.9, 300.0), (10.0, -33.0, 0.0), (179.9, 0.0, 12.0),
                                       (3.0, 80.5, -20.0), (-1.0, -89.9, 5.0), (151.2, -33.9, 40.0)])
def test_geodetic_round_trip(lon, lat, h):
    r = gc.ecef_to_geodetic(*gc.geodetic_to_ecef(lon, lat, h))
    assert abs(r[0] - lon) < 1e-11 and abs(r[1] - lat) < 1e-11 and abs(r[2] - h) < 1e-6


def _meridian_arc(lat_deg):
    a, f = gc.WGS84_A, gc.WGS84_F
    e2 = f * (2 - f)
    x = np.linspace(0.0, math.radians(lat_deg), 200001)
    y = a * (1 - e2) / (1 - e2 * np.sin(x) ** 2) ** 1.5
    hs = x[1] - x[0]
    return hs / 3 * (y[0] + y[-1] + 4 * y[1:-1:2].sum() + 2 * y[2:-1:2].sum())


@pytest.mark.parametrize("lat", [0.5, 30.0, 46.9, 60.0, 84.0])
def test_utm_on_the_central_meridian(lat):
    e, n = gc.utm_forward(-93.0, lat, 32615)          # zone 15: central meridian 93 W
    assert abs(e - 500000.0) < 1e-6
    assert abs(n - gc.UTM_K0 * _meridian_arc(lat)) < 1e-6
    es, ns = gc.utm_forward(-93.0, -lat, 32715)
    assert abs(es - 500000.0) < 1e-6 and abs(ns - (10000000.0 - gc.UTM_K0 * _meridian_arc(lat))) < 1e-6


@pytest.mark.parametrize("lon,lat", [(-95.3, 46.9), (-90.1, 10.0), (14.9, -40.0)])
def test_utm_is_conformal(lon, lat):
    epsg = 32600 + int((lon + 180) // 6) + 1 if lat >= 0 else 32700 + int((lon + 180) // 6) + 1
    d = 1e-6
    p0 = np.array(gc.utm_forward(lon, lat, epsg))
    dl = np.array(gc.utm_forward(lon + d, lat, epsg)) - p0
    dp = np.array(gc.utm_forward(lon, lat + d, epsg)) - p0
    a, f = gc.WGS84_A, gc.WGS84_F
    e2 = f * (2 - f)
    s = math.sin(math.radians(lat))
    nn, mm = a / math.sqrt(1 - e2 * s * s), a * (1 - e2) / (1 - e2 * s * s) ** 1.5
    kx = np.linalg.norm(dl) / (nn * math.cos(math.radians(lat)) * math.radians(d))
    ky = np.linalg.norm(dp) / (mm * math.radians(d))
    assert abs(kx - ky) < 1e-7 and abs(np.dot(dl, dp)) / (np.linalg.norm(dl) * np.linalg.norm(dp)) < 1e-7
    assert 0.9995 < kx < 1.001


def test_auto_zone_follows_the_reference_rule():
    assert gc.utm_epsg_auto(gc.geodetic_to_ecef(-96.8, 46.9, 0.0)) == 32614
    assert gc.utm_epsg_auto(gc.geodetic_to_ecef(151.2, -33.9, 0.0)) == 32756
    assert gc.utm_epsg_auto(gc.geodetic_to_ecef(-180.0 + 1e-9, 1.0, 0.0)) == 32601


def _scene_geo():
    c = gc.geodetic_to_ecef(-96.8, 46.9, 270.0)
    lon, lat = math.radians(-96.8), math.radians(46.9)
    east = np.array([-math.sin(lon), math.cos(lon), 0.0])
    north = np.array([-math.sin(lat) * math.cos(lon), -math.sin(lat) * math.sin(lon), math.cos(lat)])
    th = math.radians(20.0)                          # image plane axes rotated against east/north
    uiax, uiay = math.cos(th) * east + math.sin(th) * north, -math.sin(th) * east + math.cos(th) * north
    geo = {"dr": 0.21, "dc": 0.19, "dhat": (0.96, 0.28), "chat": (-0.28, 0.96)}
    return c, uiax, uiay, geo


@pytest.mark.parametrize("flip_col,flip_row", [(False, False), (True, False), (False, True)])
def test_affine_matches_reference_arithmetic(flip_col, flip_row):
    c, uiax, uiay, geo = _scene_geo()
    epsg, aff = gc.geotransform((8192, 8192), geo, c, uiax, uiay, "auto", flip_col, flip_row)
    assert epsg == 32614
    ref = geotiff_ref.affine((8192, 8192), geo, c, uiax, uiay, lambda p: gc.ecef_to_utm(p, epsg), flip_col, flip_row)
    assert np.allclose(aff, ref, rtol=0, atol=1e-9)
    # the centre pixel maps to the scene centre; pixel steps are about the ground spacing (UTM scale ~ 1)
    x = aff[0] * 4096 + aff[1] * 4096 + aff[2]
    y = aff[3] * 4096 + aff[4] * 4096 + aff[5]
    assert np.allclose((x, y), gc.ecef_to_utm(c, epsg), atol=1e-6)
    assert abs(math.hypot(aff[0], aff[3]) - 0.21) < 1e-3 and abs(math.hypot(aff[1], aff[4]) - 0.19) < 1e-3


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float32])
def test_geotiff_round_trip(tmp_path, dtype):
    Image = pytest.importorskip("PIL.Image")
    d = (np.random.default_rng(1).random((150, 97)) * 250).astype(dtype)
    aff = (0.2, -0.07, 612345.5, 0.07, -0.2, 5195432.25)
    path = gc.write_geotiff(tmp_path / "x.tif", d, 32614, aff)
    im = Image.open(path)
    assert np.array_equal(np.array(im), d)
    mt = im.tag_v2[34264]
    assert mt[:8] == (aff[0], aff[1], 0.0, aff[2], aff[3], aff[4], 0.0, aff[5])
    assert im.tag_v2[34735][-1] == 32614
