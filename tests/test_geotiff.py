"""GeoTIFF export (write_geotiff / save_maps without GDAL): pixels, orientation
and georeferencing tags, read back with PIL and with a minimal TIFF parser."""
import struct
import types

import numpy as np
import pytest
from PIL import Image

from slm_b200 import geotiff as G


def _parse(path):
    """IFD tags {tag: (type, count, raw value bytes)} and the strip bytes."""
    b = open(path, "rb").read()
    assert b[:4] == b"II*\0"
    off = struct.unpack("<I", b[4:8])[0]
    n = struct.unpack("<H", b[off:off + 2])[0]
    size = {2: 1, 3: 2, 4: 4, 12: 8}
    tags = {}
    for k in range(n):
        tag, typ, count = struct.unpack("<HHI", b[off + 2 + 12 * k: off + 10 + 12 * k])
        v = b[off + 10 + 12 * k: off + 14 + 12 * k]
        nbytes = size[typ] * count
        raw = v[:nbytes] if nbytes <= 4 else b[struct.unpack("<I", v)[0]:struct.unpack("<I", v)[0] + nbytes]
        tags[tag] = (typ, count, raw)
    so = struct.unpack("<I", tags[273][2])[0]
    sc = struct.unpack("<I", tags[279][2])[0]
    return tags, b[so:so + sc]


GEO = types.SimpleNamespace(pad_width=2, roi_nx=30, roi_ny=20,
                            roi_geotransform=[500000.0, 2.0, 0.0, 4100000.0, 0.0, -2.0],
                            projection='PROJCS["WGS 84 / UTM zone 13N"]')


@pytest.mark.parametrize("dtype", ["float32", "float64", "uint8", "bool", "int16", "uint16", "int32", "uint32"])
def test_write_geotiff_pixels_orientation_and_tags(tmp_path, dtype):
    rng = np.random.default_rng(1)
    nxp, nyp = 34, 24
    a = (rng.random((nxp, nyp)) * 200).astype(dtype)
    f = str(tmp_path / "grid.tif")
    pslice = np.index_exp[2:-2, 2:-2]
    G.write_geotiff(str(tmp_path), f, a, 30, 20, 1, pslice, GEO, epsg=32613)
    expect = np.flipud(a[pslice].T)
    tags, strip = _parse(f)
    got = np.frombuffer(strip, dtype=np.uint8 if dtype == "bool" else np.dtype(dtype).newbyteorder("<"))
    assert np.array_equal(got.reshape(20, 30), expect.astype(np.uint8) if dtype == "bool" else expect)
    assert struct.unpack("<3d", tags[33550][2]) == (2.0, 2.0, 0.0)
    assert struct.unpack("<6d", tags[33922][2]) == (0.0, 0.0, 0.0, 500000.0, 4100000.0, 0.0)
    keys = struct.unpack("<%dH" % tags[34735][1], tags[34735][2])
    assert keys[:4] == (1, 1, 0, 4) and (3072, 0, 1, 32613) == keys[16:20]
    assert tags[34737][2].rstrip(b"\0").decode() == GEO.projection + "|"
    if dtype in ("float32", "uint8", "bool", "int32", "uint16"):
        im = np.asarray(Image.open(f))
        assert np.array_equal(im, expect.astype(np.uint8) if dtype == "bool" else expect)


def test_rotated_geotransform_uses_model_transformation(tmp_path):
    f = str(tmp_path / "rot.tif")
    G.write_tiff(f, np.zeros((3, 4), np.float32), (10.0, 1.0, 0.5, 20.0, 0.25, -1.0))
    tags, _ = _parse(f)
    assert 33550 not in tags and struct.unpack("<16d", tags[34264][2])[:8] == (1.0, 0.5, 0.0, 10.0,
                                                                              0.25, -1.0, 0.0, 20.0)


def test_save_maps_writes_padded_roi_grids(tmp_path):
    nxp, nyp = 34, 24
    trace = types.SimpleNamespace(slt_array=np.ones((nxp, nyp, 2), np.float32),  # 2 values per pixel: skipped
                                  hsl_array=np.arange(nxp * nyp, dtype=np.float32).reshape(nxp, nyp),
                                  mask_array=np.zeros((nxp, nyp), bool), other=np.zeros((5, 5)),
                                  count_array=np.ones((nxp, nyp, 1), np.uint32))
    files = G.save_maps([trace], GEO, str(tmp_path / "job"))
    assert sorted(f.rsplit("/", 1)[1] for f in files) == ["job_count.tif", "job_hsl.tif", "job_mask.tif"]
    im = np.asarray(Image.open(str(tmp_path / "job_hsl.tif")))
    assert np.array_equal(im, np.flipud(trace.hsl_array[2:-2, 2:-2].T))
