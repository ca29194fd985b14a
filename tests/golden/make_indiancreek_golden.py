#!/usr/bin/env python3
"""Write tests/golden/indiancreek_test2.npz from the reference's own data.

The reference's IndianCreek Test#2 job (tests/IndianCreek_Test2.json) reads
data/IndianCreek_res1m_fillsinks0p01_cuttest2.tif (a 200 x 200 float32 DTM at
1 m) and data/IndianCreek_DTM0_res1m_fill_sinks1deg_watershed3k_cuttest2.tif
(basin indexes), and keeps basins 1131 and 1132.  This script reads both with
PIL (no GDAL here) and stores what the reference's Geodata stage makes of
them (geodata.py:95-250):

* ``roi``: the DTM as the ROI array, ``flipud(dtm).T`` (x-major, y north
  up), with the no-data values of json/defaults.json (-99999 and 0) as NaN;
* ``basin_mask``: True outside basins 1131/1132, in the same orientation
  (unpadded; the stages pad it with True).

The reference checkout is ``$SLM_REFERENCE``, else ``reference`` beside this
repository.  The fixture is small (two 200 x 200 grids) and travels with the
repository to hosts without the checkout.
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_REF = os.environ.get("SLM_REFERENCE") or os.path.join(
    os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference")
OUT = os.path.join(HERE, "indiancreek_test2.npz")
DTM = "IndianCreek_res1m_fillsinks0p01_cuttest2.tif"
BASINS = "IndianCreek_DTM0_res1m_fill_sinks1deg_watershed3k_cuttest2.tif"
KEEP = (1131, 1132)
NO_DATA = (-99999.0, 0.0)


def read_tif(path):
    from PIL import Image
    return np.array(Image.open(path), dtype=np.float32)


def make(reference=DEFAULT_REF, out=OUT):
    data = os.path.join(reference, "data")
    dtm = read_tif(os.path.join(data, DTM))
    for v in NO_DATA:
        dtm[dtm == v] = np.nan
    basins = read_tif(os.path.join(data, BASINS))
    roi = np.flipud(dtm).T.copy()
    keep = np.isin(np.flipud(basins).T, KEEP)
    np.savez_compressed(out, roi=roi.astype(np.float32), basin_mask=~keep, pixel_size=np.float32(1.0),
                        basins=np.array(KEEP))
    return out


if __name__ == "__main__":
    print(make())
