"""Oracle (test infrastructure only): the fast-marching signed distance that
the reference's pass 2 takes from scikit-fmm (``skfmm.distance``), restated.

Only ``tests/`` use this file, as the checker of ``slm_fmm_lengths``
(``slm_b200/csrc/fmm.cu``) and as a stand-in for ``skfmm`` when the
reference's own ``Mapping.fmm_lengths`` (python/streamlines/mapping.py:841-900)
runs in a test.  Nothing in the product path imports it.

Parity unpinned: scikit-fmm (PyPI ``scikit-fmm``; the reference pins no
version) is not installed here and has no golden vectors in the reference,
so what follows is this project's restatement of the published method, not a
reproduction of that library's arithmetic:

* the fast marching method of J. A. Sethian (PNAS 93, 1996; "Level Set
  Methods and Fast Marching Methods", 1999, ch. 8), on a 2-D grid of unit
  spacing, the distance multiplied by ``dx`` at the end;
* the zero contour is located by linear interpolation between each point
  and its axis neighbours of the other sign: along an axis the distance is
  |phi_p| / |phi_p - phi_q| (the nearer side), and a point with crossings on
  both axes takes 1 / sqrt(1/dx^2 + 1/dy^2) -- the interface treated as a
  straight line through the two crossings.  These points are frozen first;
* the upwind update on |distance|: per axis the frozen neighbour of
  smaller value a (the lower-index side on a tie), with Sethian's
  second-order one-sided difference (3u - 4a + b) / 2 when the next point b
  on that side is frozen and b <= a (``order`` 2, scikit-fmm's default),
  else the first-order (u - a).  A frozen value across the contour enters
  with its sign flipped (the signed distance is continuous there), so a
  second-order stencil that reaches over the contour stays exact for a
  straight one.  The quadratic over both axes is taken when
  its root is at least both axes' a, else the axis of smaller a alone;
* points are frozen in increasing (distance, row-major index) order, so the
  result does not depend on how the narrow band is stored;
* masked points are neither computed nor used; unmasked points that no
  front reaches are masked in the result.  A grid without a zero contour
  raises ValueError (as scikit-fmm does).

Every arithmetic step below is an IEEE double operation in a fixed order;
the CUDA kernel performs the same operations in the same order (compiled
with --fmad=false), so the two agree bit for bit.
"""
from __future__ import annotations

import heapq
import math

import numpy as np

FAR, BAND, FROZEN = 0, 1, 2


def _rel(val, neg, x, y, qx, qy):
    """The frozen |distance| at q as seen from p's side of the contour:
    negative across it (the signed distance is continuous there)."""
    v = val[qx, qy]
    return -v if neg[x, y] != neg[qx, qy] else v


def _axis_term(val, neg, state, unmasked, nx, ny, x, y, dx_, dy_, order):
    """(a, alpha, beta) of one axis at (x, y), or None without a frozen
    neighbour.  The minus side wins a tie."""
    best = None
    for s in (-1, 1):
        qx, qy = x + s * dx_, y + s * dy_
        if 0 <= qx < nx and 0 <= qy < ny and unmasked[qx, qy] and state[qx, qy] == FROZEN:
            a = _rel(val, neg, x, y, qx, qy)
            if best is None or a < best[0]:
                best = (a, s)
    if best is None:
        return None
    a, s = best
    if order == 2:
        rx, ry = x + 2 * s * dx_, y + 2 * s * dy_
        if 0 <= rx < nx and 0 <= ry < ny and unmasked[rx, ry] and state[rx, ry] == FROZEN:
            b = _rel(val, neg, x, y, rx, ry)
            if b <= a:
                return (a, 1.5, (4.0 * a - b) / 2.0)
    return (a, 1.0, a)


def _update(val, neg, state, unmasked, nx, ny, x, y, order):
    """The tentative |distance| of (x, y) from its frozen neighbours (pixel units)."""
    t0 = _axis_term(val, neg, state, unmasked, nx, ny, x, y, 1, 0, order)
    t1 = _axis_term(val, neg, state, unmasked, nx, ny, x, y, 0, 1, order)
    if t0 is None and t1 is None:
        return None
    if t0 is not None and t1 is not None:
        lo, hi = (t0, t1) if t0[0] <= t1[0] else (t1, t0)
        A = lo[1] * lo[1] + hi[1] * hi[1]
        B = lo[1] * lo[2] + hi[1] * hi[2]
        C = (lo[2] * lo[2] + hi[2] * hi[2]) - 1.0
        disc = B * B - A * C
        if disc >= 0.0:
            u = (B + math.sqrt(disc)) / A
            if u >= hi[0]:
                return u
        one = lo
    else:
        one = t0 if t0 is not None else t1
    return (one[2] + 1.0) / one[1]


def distance_unit(phi, unmasked, order=2):
    """Signed distance in pixel units from the zero contour of ``phi``
    (float64 [nx, ny]) over the ``unmasked`` points; returns (dist, reached).
    Raises ValueError when there is no zero contour."""
    phi = np.asarray(phi, dtype=np.float64)
    unmasked = np.asarray(unmasked, dtype=bool)
    nx, ny = phi.shape
    val = np.zeros((nx, ny), dtype=np.float64)
    state = np.zeros((nx, ny), dtype=np.uint8)
    neg = phi < 0.0
    n_frozen = 0
    for x in range(nx):
        for y in range(ny):
            if not unmasked[x, y]:
                continue
            p = phi[x, y]
            if p == 0.0:
                state[x, y] = FROZEN
                val[x, y] = 0.0
                n_frozen += 1
                continue
            inv = 0.0
            crossed = False
            for dx_, dy_ in ((1, 0), (0, 1)):
                dmin = None
                for s in (-1, 1):
                    qx, qy = x + s * dx_, y + s * dy_
                    if 0 <= qx < nx and 0 <= qy < ny and unmasked[qx, qy]:
                        q = phi[qx, qy]
                        if (p > 0.0 and q < 0.0) or (p < 0.0 and q > 0.0):
                            d = abs(p) / abs(p - q)
                            if dmin is None or d < dmin:
                                dmin = d
                if dmin is not None:
                    inv = inv + 1.0 / (dmin * dmin)
                    crossed = True
            if crossed:
                state[x, y] = FROZEN
                val[x, y] = 1.0 / math.sqrt(inv)
                n_frozen += 1
    if n_frozen == 0:
        raise ValueError("the array phi contains no zero contour (no zero level set)")
    heap = []
    for x in range(nx):
        for y in range(ny):
            if unmasked[x, y] and state[x, y] == FAR:
                u = _update(val, neg, state, unmasked, nx, ny, x, y, order)
                if u is not None:
                    val[x, y] = u
                    state[x, y] = BAND
                    heap.append((u, x * ny + y))
    heapq.heapify(heap)
    while heap:
        u, i = heapq.heappop(heap)
        x, y = divmod(i, ny)
        if state[x, y] == FROZEN or u != val[x, y]:
            continue
        state[x, y] = FROZEN
        for qx, qy in ((x - 1, y), (x + 1, y), (x, y - 1), (x, y + 1)):
            if 0 <= qx < nx and 0 <= qy < ny and unmasked[qx, qy] and state[qx, qy] != FROZEN:
                w = _update(val, neg, state, unmasked, nx, ny, qx, qy, order)
                if state[qx, qy] == FAR or w != val[qx, qy]:
                    val[qx, qy] = w
                    state[qx, qy] = BAND
                    heapq.heappush(heap, (w, qx * ny + qy))
    reached = unmasked & (state == FROZEN)
    sign = np.where(neg, -1.0, 1.0)
    return np.where(reached, sign * val, 0.0), reached


def distance(phi, dx=1.0, order=2):
    """``skfmm.distance``'s call form: ``phi`` a float array or a NumPy
    masked array (masked points excluded); returns a masked array of the
    signed distance times ``dx`` (masked where phi is masked or unreached)."""
    if isinstance(phi, np.ma.MaskedArray):
        data = np.asarray(phi.data, dtype=np.float64)
        unmasked = ~np.ma.getmaskarray(phi)
    else:
        data = np.asarray(phi, dtype=np.float64)
        unmasked = np.ones(data.shape, dtype=bool)
    d, reached = distance_unit(data, unmasked, order)
    return np.ma.MaskedArray(d * float(dx), mask=~reached)


def solve_problems(label, flags, thin_bit, subsegments, dx, order, fields=False):
    """The oracle of ``slm_fmm_lengths`` / ``slm_b200.fmm.device_solver``:
    per |label| value in ``subsegments``, phi on the whole window as the
    reference's ``fmm_lengths`` builds it (own pixels grown by one with the
    4-neighbour structure are the domain; own thin-channel pixels -1, the
    rest +1), the distance above, and (sum, count, n_phi, n_channel,
    status) with the sum taken over the reached pixels in row-major order.
    ``label`` / ``flags`` are NumPy [nx, ny] arrays (or tensors)."""
    from scipy.ndimage import binary_dilation, generate_binary_structure
    label = np.asarray(label.cpu().numpy() if hasattr(label, "cpu") else label).astype(np.int64)
    flags = np.asarray(flags.cpu().numpy() if hasattr(flags, "cpu") else flags).astype(np.int64) & 0xFFFFFFFF
    keys = np.asarray(subsegments, dtype=np.int64)
    n = keys.shape[0]
    out = [np.zeros(n, np.float64), np.zeros(n, np.int64), np.zeros(n, np.int64), np.zeros(n, np.int64),
           np.full(n, 1, np.int32)]
    per = [None] * n
    thin = int(thin_bit) & 0xFFFFFFFF
    for i, s in enumerate(keys):
        own = np.abs(label) == s
        if not own.any():
            continue
        dom = binary_dilation(own, structure=generate_binary_structure(2, 1), iterations=1)
        chan = own & ((flags & thin) == thin)
        out[2][i], out[3][i] = int(own.sum()), int(chan.sum())
        if out[3][i] == 0:
            continue
        phi = np.where(chan, -1.0, 1.0)
        try:
            d, reached = distance_unit(phi, dom, order)
        except ValueError:
            out[4][i] = 2
            continue
        dist = np.where(reached, d, 0.0) * float(dx)
        acc = 0.0
        for v in dist[reached]:  # row-major order
            acc = acc + float(v)
        out[0][i], out[1][i], out[4][i] = acc, int(reached.sum()), 0
        per[i] = (dist, reached)
    return tuple(out) + ((per,) if fields else ())
