"""CPU restatement of the reference's DTM preprocessing (test infrastructure).

This is the oracle for ``slm_preprocess``: it restates, in NumPy, the
conditioned gradient vector field of python/streamlines/preprocess.py.  Only
tests, the smoke check and the bench's CPU leg use it.

Steps, each citing the reference lines it follows:

- ``blockage_codes``: find_blockages' first generic_filter
  (preprocess.py:647-667) with has_one_diagonal_outflow (:389-431).  The
  filter runs over roi.T with size 3 and scipy's default 'reflect' mode, which
  for a 3x3 window repeats the edge pixel (clamped indices).
- ``blocked_neighbor_codes``: the second generic_filter (:668-671) with
  upstream_of_diagonal_outflow (:433-477) on the codes.
- ``gradient_velocity``: compute_topo_gradient_field (:51-63, np.gradient
  on the float32 ROI, one-sided at the edges, then / pixel_size in float32)
  and compute_gradient_velocity_field (:176-193: negate, speed = hypot with
  non-finite or zero speeds set to 1, normalise).
- ``loop_cells``: find_and_fix_loops' detection (:302-340) with
  check_has_loop (:228-260) as numba compiles it: the mean velocity's sums
  in float32, its speed in double (``velocity / 4.0`` is a float64 array
  there) rounded to float32, divergence and curl in float32; thresholds
  compare in double (a float32 against a float64 parameter).  Cells in the last row
  or column read one pixel beyond the grid in the reference (undefined
  there); none of the pixels they mark is far enough inside the grid to be
  fixed, so they are skipped here.
- ``fix_loops``: break_out_of_loop (:262-300) for every marked pixel: the
  lowest of the 8 neighbours (first in W, E, S, N, SW, SE, NW, NE order on
  ties) sets a unit vector, component / hypot in float32 (numba picks the
  float32 loop of np.hypot for int8 arguments).
- ``fix_blockages`` (:351-387): blockages, then blocked neighbours, set
  (dx, dy) / sqrt(2) of their code's flow vector (get_flow_vector :195-226).
- the final normalisation or un-normalisation (:588-592), edge padding
  (:594-598), slope (:597-598) and mask_nan_uv (:602-621).
"""
from __future__ import annotations

import numpy as np

# get_flow_vector (preprocess.py:195-226): priority SW, SE, NW, NE, W, E, S, N
_FLOW_ORDER = ((16, -1, -1), (32, +1, -1), (64, -1, +1), (128, +1, +1),
               (1, -1, 0), (2, +1, 0), (4, 0, -1), (8, 0, +1))
# break_out_of_loop's vec_list: get_flow_vector of 1, 2, 4, ..., 128
_BREAK_VECS = ((-1, 0), (+1, 0), (0, -1), (0, +1), (-1, -1), (+1, -1), (-1, +1), (+1, +1))
_INV_SQRT2_F32 = np.float32(np.float32(1.0) / np.sqrt(2.0))


def flow_vector(code):
    for bit, dx, dy in _FLOW_ORDER:
        if code & bit:
            return dx, dy
    return 0, 0


def _clamped_window(a):
    """Neighbour views a[x+dx, y+dy] with clamped indices, keyed (dx, dy)."""
    p = np.pad(a, 1, mode="edge")
    nx, ny = a.shape
    return {(dx, dy): p[1 + dx:1 + dx + nx, 1 + dy:1 + dy + ny] for dx in (-1, 0, 1) for dy in (-1, 0, 1)}


def blockage_codes(roi):
    """has_one_diagonal_outflow over the clamped 3x3 window: the bit set of
    lower neighbours when all of them are diagonal, else 0.  roi is [nx, ny]
    (x-major); the window's (dx, dy) offsets are the reference's compass
    points: S is -y, W is -x."""
    w = _clamped_window(np.asarray(roi))
    h = w[(0, 0)]
    nn = np.zeros(h.shape, np.uint8)
    for (dx, dy), bit in (((-1, -1), 16), ((0, -1), 4), ((1, -1), 32), ((-1, 0), 1), ((1, 0), 2),
                          ((-1, 1), 64), ((0, 1), 8), ((1, 1), 128)):
        nn |= np.where(w[(dx, dy)] < h, np.uint8(bit), np.uint8(0))
    return np.where((nn & 0xF0) == nn, nn, np.uint8(0)).astype(np.uint8)


def blocked_neighbor_codes(codes):
    """upstream_of_diagonal_outflow over the clamped 3x3 window of codes."""
    w = _clamped_window(np.asarray(codes))
    nn = np.zeros(codes.shape, np.uint8)
    rules = (((-1, -1), (16,), 16), ((0, -1), (16, 32), 4), ((1, -1), (32,), 32), ((-1, 0), (16, 64), 1),
             ((1, 0), (128, 32), 2), ((-1, 1), (64,), 64), ((0, 1), (64, 128), 8), ((1, 1), (128,), 128))
    for off, matches, bit in rules:
        hit = np.zeros(codes.shape, bool)
        for m in matches:
            hit |= w[off] == m
        nn |= np.where(hit, np.uint8(bit), np.uint8(0))
    return nn


def hypot_f32(u, v):
    """np.hypot of float32 arrays: the double sum of the exact squares,
    square-rooted and rounded to float32 (identical to the C library's
    hypotf on this platform's NumPy)."""
    return np.hypot(np.asarray(u, np.float32), np.asarray(v, np.float32))


def speed_field(u, v):
    """set_speed_field (preprocess.py:118-136)."""
    s = hypot_f32(u, v)
    s[(~np.isfinite(s)) | (s == 0.0)] = np.float32(1.0)
    return s


def gradient_velocity(roi, pixel_size):
    """(u, v, raw_speed) float32 [nx, ny] of compute_gradient_velocity_field."""
    f = np.asarray(roi).astype(np.float32)
    ps = np.float32(pixel_size)
    gx = np.gradient(f, axis=0) / ps
    gy = np.gradient(f, axis=1) / ps
    u, v = -gx, -gy
    speed = speed_field(u, v)
    return u / speed, v / speed, speed, gx, gy


def loop_cells(u, v, vecsum_threshold=0.95, divergence_threshold=-0.5, curl_threshold=0.0):
    """uint8 [nx, ny]: 1 at cell (x, y) (pixels x..x+1, y..y+1) when
    check_has_loop's speed, divergence and curl pass the three thresholds."""
    nx, ny = u.shape
    out = np.zeros((nx, ny), np.uint8)
    if nx < 2 or ny < 2:
        return out
    u00, u10, u11, u01 = u[:-1, :-1], u[1:, :-1], u[1:, 1:], u[:-1, 1:]
    v00, v10, v11, v01 = v[:-1, :-1], v[1:, :-1], v[1:, 1:], v[:-1, 1:]
    f = np.float32
    vx = (((u00 + u10) + u11) + u01) / f(4.0)
    vy = (((v00 + v10) + v11) + v01) / f(4.0)
    # numba types `velocity / 4.0` as float64, so the speed is the double
    # sqrt of the double dot product, rounded to float32 (= hypot_f32)
    speed = hypot_f32(vx, vy)
    div = (((-u00 - v00) + (u10 - v10)) + (u11 + v11)) + (-u01 + v01)
    curl = (((u00 - v00) + (u10 + v10)) + (-u11 + v11)) + (-u01 - v01)
    with np.errstate(invalid="ignore"):
        hit = ((speed.astype(np.float64) < float(vecsum_threshold))
               & (div.astype(np.float64) <= float(divergence_threshold))
               & (np.abs(curl).astype(np.float64) >= float(curl_threshold)))
    out[:-1, :-1] = hit
    return out


def looped_pixels(cells):
    """Pixels marked by any looped cell (the cell's four corners)."""
    m = cells.astype(bool)
    p = m.copy()
    p[1:, :] |= m[:-1, :]
    p[:, 1:] |= m[:, :-1]
    p[1:, 1:] |= m[:-1, :-1]
    return p


def break_vector(roi, x, y):
    """break_out_of_loop's unit vector at a pixel well inside the grid."""
    h_min = np.float64(np.finfo(np.float32).max)
    best = 0
    for k, (dx, dy) in enumerate(_BREAK_VECS):
        h = roi[x + dx, y + dy]
        if h_min > h:
            h_min = h
            best = k
    dx, dy = _BREAK_VECS[best]
    n = np.float32(np.hypot(np.float32(dx), np.float32(dy)))
    return np.float32(np.float32(dx) / n), np.float32(np.float32(dy) / n)


def break_vectors(roi, marked):
    """break_vector for every marked pixel well inside the grid, vectorised:
    (mask of fixed pixels, u, v).  The first strict minimum below FLT_MAX
    wins, as in the reference's scan; NaN and values >= FLT_MAX never do."""
    nx, ny = roi.shape
    fix = np.zeros((nx, ny), bool)
    fix[1:-1, 1:-1] = marked[1:-1, 1:-1]
    xs, ys = np.nonzero(fix)
    fmax = np.float64(np.finfo(np.float32).max)
    h = np.stack([roi[xs + dx, ys + dy].astype(np.float64) for dx, dy in _BREAK_VECS], axis=1)
    h = np.where(h < fmax, h, np.inf)  # NaN compares false: never lower
    best = np.argmin(h, axis=1)  # first minimum; all-inf rows give 0 (W)
    vec = np.array(_BREAK_VECS, np.float32)[best]
    n = np.hypot(vec[:, 0], vec[:, 1]).astype(np.float32)
    return fix, xs, ys, (vec[:, 0] / n).astype(np.float32), (vec[:, 1] / n).astype(np.float32)


def flow_vectors(codes):
    """get_flow_vector over an array of codes: (dx, dy) int arrays."""
    conds = [(codes & bit) != 0 for bit, _, _ in _FLOW_ORDER]
    dx = np.select(conds, [d for _, d, _ in _FLOW_ORDER], 0)
    dy = np.select(conds, [d for _, _, d in _FLOW_ORDER], 0)
    return dx, dy


def conditioned_uv(roi, pixel_size, pad_width, vecsum_threshold=0.95, divergence_threshold=-0.5,
                   curl_threshold=0.0, do_normalize_speed=True):
    """The whole conditioned preprocess of one ROI; a dict of its arrays."""
    roi = np.asarray(roi)
    codes = blockage_codes(roi)
    nbr = blocked_neighbor_codes(codes)
    u, v, raw_speed, gx, gy = gradient_velocity(roi, pixel_size)
    cells = loop_cells(u, v, vecsum_threshold, divergence_threshold, curl_threshold)
    u, v = u.copy(), v.copy()
    _, xs, ys, bu, bv = break_vectors(roi, looped_pixels(cells))
    u[xs, ys], v[xs, ys] = bu, bv
    for arr in (codes, nbr):
        xs, ys = np.nonzero(arr)
        dx, dy = flow_vectors(arr[xs, ys])
        u[xs, ys] = np.where(dx != 0, dx.astype(np.float32) * _INV_SQRT2_F32, np.float32(0.0))
        v[xs, ys] = np.where(dy != 0, dy.astype(np.float32) * _INV_SQRT2_F32, np.float32(0.0))
    if do_normalize_speed:
        s = speed_field(u, v)
        u, v = u / s, v / s
    else:
        u, v = u * raw_speed, v * raw_speed
    pw = int(pad_width)
    uv = np.stack((np.pad(u, pw, "edge"), np.pad(v, pw, "edge")), axis=2).astype(np.float32)
    slope = np.rad2deg(np.arctan(np.pad(raw_speed, pw, "edge"))).astype(np.float32)
    uv_mask = np.isnan(uv[:, :, 0]) | np.isnan(uv[:, :, 1])
    uv[uv_mask] = 0.0
    n_cells = int(cells.sum())
    where_looped = np.zeros((4 * n_cells, 2), np.uint32)
    cx, cy = np.nonzero(cells)
    for k, (ox, oy) in enumerate(((0, 0), (1, 0), (0, 1), (1, 1))):
        where_looped[k::4, 0] = cx + ox
        where_looped[k::4, 1] = cy + oy
    return {"uv_array": uv, "slope_array": slope, "uv_mask_array": uv_mask,
            "blockages_array": codes, "blocked_neighbors_array": nbr, "loop_cells": cells,
            "where_looped_array": where_looped, "n_loops": 4 * n_cells,
            "roi_gradx_array": gx, "roi_grady_array": gy}
