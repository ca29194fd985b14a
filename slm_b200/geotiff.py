"""GeoTIFF export of the stage grids, without GDAL.

Mirrors ``useful.write_geotiff`` (python/streamlines/useful.py:349-389) and
``Save.save_maps`` (save.py:191-231).  The reference writes each padded
[nxp, nyp] grid through GDAL:

- the ``pslice`` crop (the pad removed), transposed and flipped north-up;
- one band, of the GDAL type matching the NumPy dtype (bool as uint8);
- the ROI's geotransform and the DTM's projection.

GDAL is not available here, so this module writes the TIFF itself.  It is a
baseline little-endian TIFF with one uncompressed strip, and SampleFormat
gives the type.  The georeferencing is stored as GeoTIFF tags:

- ModelPixelScale and ModelTiepoint for a north-up geotransform, or
  ModelTransformation when the geotransform has rotation terms;
- a GeoKeyDirectory: projected model, pixel-is-area raster;
- the projection string (e.g. GDAL's WKT) as the GT citation.  GDAL reads
  that back as a citation, not as an EPSG-coded CRS; pass ``epsg`` to add
  ProjectedCSTypeGeoKey.
"""
from __future__ import annotations

import os
import struct

import numpy as np

# NumPy dtype -> (BitsPerSample, SampleFormat: 1 unsigned, 2 signed, 3 float)
_TYPES = {np.dtype("bool"): (8, 1), np.dtype("int8"): (8, 2), np.dtype("uint8"): (8, 1),
          np.dtype("int16"): (16, 2), np.dtype("uint16"): (16, 1), np.dtype("int32"): (32, 2),
          np.dtype("uint32"): (32, 1), np.dtype("float32"): (32, 3), np.dtype("float64"): (64, 3)}
_SHORT, _LONG, _DOUBLE, _ASCII = 3, 4, 12, 2
_FMT = {_SHORT: "H", _LONG: "I", _DOUBLE: "d"}


def _entries(width, height, bits, fmt, geotransform, projection, epsg):
    gt = [float(v) for v in geotransform]
    e = [(256, _LONG, [width]), (257, _LONG, [height]), (258, _SHORT, [bits]), (259, _SHORT, [1]),
         (262, _SHORT, [1]), (273, _LONG, [0]), (277, _SHORT, [1]), (278, _LONG, [height]),
         (279, _LONG, [0]), (284, _SHORT, [1]), (339, _SHORT, [fmt])]
    if gt[2] == 0.0 and gt[4] == 0.0:
        e.append((33550, _DOUBLE, [gt[1], -gt[5], 0.0]))  # ModelPixelScale
        e.append((33922, _DOUBLE, [0.0, 0.0, 0.0, gt[0], gt[3], 0.0]))  # ModelTiepoint
    else:  # ModelTransformation: 4 x 4, row major
        e.append((34264, _DOUBLE, [gt[1], gt[2], 0.0, gt[0], gt[4], gt[5], 0.0, gt[3],
                                   0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0]))
    citation = (projection or "") + "|"
    keys = [(1024, 0, 1, 1),                          # GTModelTypeGeoKey: projected
            (1025, 0, 1, 1),                          # GTRasterTypeGeoKey: pixel is area
            (1026, 34737, len(citation), 0)]          # GTCitationGeoKey -> GeoAsciiParams
    if epsg:
        keys.append((3072, 0, 1, int(epsg)))          # ProjectedCSTypeGeoKey
    directory = [1, 1, 0, len(keys)] + [v for k in keys for v in k]
    e.append((34735, _SHORT, directory))
    e.append((34737, _ASCII, citation))
    return sorted(e, key=lambda t: t[0])


def write_tiff(file_name, band, geotransform=(0.0, 1.0, 0.0, 0.0, 0.0, -1.0), projection="", epsg=None):
    """Write a 2-D array (rows north to south) as a one-band GeoTIFF."""
    band = np.ascontiguousarray(band)
    if band.ndim != 2 or band.dtype not in _TYPES:
        raise ValueError("a 2-D array of a GDAL-writable type is required, got {} {}".format(band.shape, band.dtype))
    bits, fmt = _TYPES[band.dtype]
    data = band.astype(np.uint8) if band.dtype == np.bool_ else band.astype(band.dtype.newbyteorder("<"))
    raw = data.tobytes()
    height, width = band.shape
    entries = _entries(width, height, bits, fmt, geotransform, projection, epsg)
    ifd_size = 2 + 12 * len(entries) + 4
    out_of_line = 8 + ifd_size  # values that do not fit in 4 bytes follow the IFD
    blobs, table = [], []
    for tag, typ, vals in entries:
        if typ == _ASCII:
            payload = vals.encode("ascii") + b"\0"
            count = len(payload)
        else:
            payload = struct.pack("<" + _FMT[typ] * len(vals), *vals)
            count = len(vals)
        if len(payload) <= 4:
            table.append([tag, typ, count, payload.ljust(4, b"\0"), None])
        else:
            if out_of_line % 2:
                blobs.append(b"\0")
                out_of_line += 1
            table.append([tag, typ, count, struct.pack("<I", out_of_line), None])
            blobs.append(payload)
            out_of_line += len(payload)
    data_offset = out_of_line + (out_of_line % 8 and 8 - out_of_line % 8)
    for row in table:
        if row[0] == 273:
            row[3] = struct.pack("<I", data_offset)
        elif row[0] == 279:
            row[3] = struct.pack("<I", len(raw))
    with open(file_name, "wb") as f:
        f.write(b"II*\0" + struct.pack("<I", 8))
        f.write(struct.pack("<H", len(table)))
        for tag, typ, count, value, _ in table:
            f.write(struct.pack("<HHI", tag, typ, count) + value)
        f.write(struct.pack("<I", 0))
        for b in blobs:
            f.write(b)
        f.write(b"\0" * (data_offset - out_of_line))
        f.write(raw)


def write_geotiff(path, file_name, array, nx, ny, npd, pslice, geodata, epsg=None):
    """useful.write_geotiff: the ``pslice`` crop of ``array``, transposed and
    flipped north-up, with ``geodata.roi_geotransform`` and the projection
    string ``geodata.projection`` (if any; the reference reads it from the
    DTM through GDAL).  ``path`` is unused, as in the reference."""
    if npd != 1:
        raise ValueError("one band per file, as the reference writes")
    band = np.flipud(np.asarray(array)[pslice].T)
    if band.shape != (ny, nx):
        raise ValueError("the crop is {} but nx, ny = {}, {}".format(band.shape, nx, ny))
    write_tiff(file_name, band, geodata.roi_geotransform, getattr(geodata, "projection", "") or "", epsg)


def save_maps(objects, geodata, file_stem, fmt="tif", epsg=None):
    """Save.save_maps: every 2-D array attribute of ``objects`` shaped like the
    padded ROI [nxp, nyp], cropped of its pad, as ``<file_stem>_<name>.tif``
    (the name without its ``_array`` suffix).  Returns the files written."""
    pad = geodata.pad_width
    nx, ny = geodata.roi_nx, geodata.roi_ny
    pslice = np.index_exp[pad:-pad, pad:-pad] if pad else np.index_exp[:, :]
    written = []
    for obj in objects:
        for item, ref in vars(obj).items():
            if isinstance(ref, np.ndarray) and ref.ndim == 3 and ref.shape[2] == 1:
                ref = ref[:, :, 0]  # one value per pixel: written, as the reference's npd == 1
            if isinstance(ref, np.ndarray) and ref.ndim == 2 and ref.shape == (nx + 2 * pad, ny + 2 * pad) \
                    and ref.dtype in _TYPES:
                name = "{}_{}.{}".format(file_stem, item.replace("_array", ""), fmt)
                write_geotiff(os.path.dirname(name), name, ref, nx, ny, 1, pslice, geodata, epsg)
                written.append(name)
    return written
