"""CPU restatement of the seam a source chain adds between two sources: test infrastructure only.

The product never imports this module; tests/ use it as the checker of the seam fixtures (the
reference's own fields, tests/golden/seams.npz) and of the device seam solve.

It follows detail::BuildSeamField (src/sources/seam_field.cpp:663-710) from the lattice's samples
(`data` 1 where the earlier source has data, `difference` earlier minus later, NaN elsewhere):

  - band(): NearGaps with radius 3 (seam_field.cpp:117-148) and the band's fixed differences;
  - distances(): DataDistances' two-pass chamfer relaxation in float, with the carried values
    (seam_field.cpp:151-213), as plain Python loops (small lattices only);
  - feather(): Feather's smoothstep fade (seam_field.cpp:218-241);
  - solve(): the Height / Slope system - B = -Laplacian + 1/L^2 on 5 points, or B applied twice
    on 13 points, over the gap posts within 3 decay lengths and 3 posts off the lattice's
    border, the posts around them fixed (seam_field.cpp:389-407, 597-617, 696-709) - solved
    directly (scipy.sparse), where the reference runs multigrid-preconditioned conjugate
    gradients to a residual of 1e-10.
"""

from __future__ import annotations

import math

import numpy as np

BAND_POSTS = 3    # seam_field.cpp:29
BORDER_POSTS = 3  # seam_field.cpp:32
REACH_DECAYS = 3.0  # SeamReach: the Height / Slope solve reaches 3 decay lengths


def band(data: np.ndarray, difference: np.ndarray, radius: int = BAND_POSTS) -> np.ndarray:
    """The field after the band: posts with data within `radius` posts (along both axes) of a
    post without data hold their difference; 0 elsewhere."""
    h, w = data.shape
    gap = (data == 0)
    across = np.zeros_like(gap)
    for d in range(-radius, radius + 1):
        lo, hi = max(0, d), min(w, w + d)
        across[:, lo - d:hi - d] |= gap[:, lo:hi]
    near = np.zeros_like(gap)
    for d in range(-radius, radius + 1):
        lo, hi = max(0, d), min(h, h + d)
        near[lo - d:hi - d, :] |= across[lo:hi, :]
    keep = (data != 0) & near & ~np.isnan(difference)
    return np.where(keep, difference, np.float32(0.0)).astype(np.float32)


def distances(data: np.ndarray, dx: float, dy: float, carried: np.ndarray | None = None):
    """Chamfer distances (float32) from each post to the nearest post with data and, with
    `carried` (the value at each post with data), the value carried from that post."""
    h, w = data.shape
    f32 = np.float32
    sx, sy = f32(dx), f32(dy)
    sd = f32(math.hypot(dx, dy))
    dist = np.where(data != 0, f32(0.0), f32(np.inf)).astype(np.float32).ravel().tolist()
    carry = (np.where(data != 0, carried, f32(0.0)).astype(np.float32).ravel().tolist()
             if carried is not None else None)
    has = (data != 0).ravel().tolist()
    # Python floats are doubles: each sum is rounded back to float32, as the reference's float
    # arithmetic does (a distance plus a step, both floats of like magnitude, is exact in
    # double before that rounding).
    r32 = lambda v: float(f32(v))  # noqa: E731

    def relax(to, frm, step):
        through = r32(dist[frm] + step)
        if through < dist[to]:
            dist[to] = through
            if carry is not None:
                carry[to] = carry[frm]

    fx, fy, fd = float(sx), float(sy), float(sd)
    for row in range(h):
        for col in range(w):
            k = row * w + col
            if has[k]:
                continue
            if col > 0:
                relax(k, k - 1, fx)
            if row > 0:
                relax(k, k - w, fy)
                if col > 0:
                    relax(k, k - w - 1, fd)
                if col + 1 < w:
                    relax(k, k - w + 1, fd)
    for row in range(h - 1, -1, -1):
        for col in range(w - 1, -1, -1):
            k = row * w + col
            if has[k]:
                continue
            if col + 1 < w:
                relax(k, k + 1, fx)
            if row + 1 < h:
                relax(k, k + w, fy)
                if col + 1 < w:
                    relax(k, k + w + 1, fd)
                if col > 0:
                    relax(k, k + w - 1, fd)
    d = np.array(dist, np.float32).reshape(h, w)
    c = np.array(carry, np.float32).reshape(h, w) if carry is not None else None
    return d, c


def feather(data: np.ndarray, difference: np.ndarray, dx: float, dy: float,
            width: float) -> np.ndarray:
    field = band(data, difference)
    d, carried = distances(data, dx, dy, field)
    sel = (data == 0) & (d.astype(np.float64) < width)
    t = d.astype(np.float64) / width
    weight = 1.0 - t * t * (3.0 - 2.0 * t)
    out = field.copy()
    out[sel] = (weight * carried.astype(np.float64))[sel].astype(np.float32)
    return out


def unknowns(data: np.ndarray, distance: np.ndarray, reach: float) -> np.ndarray:
    h, w = data.shape
    inside = np.zeros((h, w), bool)
    inside[BORDER_POSTS:h - BORDER_POSTS, BORDER_POSTS:w - BORDER_POSTS] = True
    return (data == 0) & inside & (distance.astype(np.float64) <= reach)


def _stencil(order: int, dx: float, dy: float, screening: float) -> dict:
    """The operator's weights by offset (dc, dr): B, or B applied twice."""
    cx, cy = 1.0 / (dx * dx), 1.0 / (dy * dy)
    c0 = 2.0 * cx + 2.0 * cy + screening
    if order == 1:
        return {(0, 0): c0, (-1, 0): -cx, (1, 0): -cx, (0, -1): -cy, (0, 1): -cy}
    s = {(0, 0): c0 * c0 + 2.0 * cx * cx + 2.0 * cy * cy}
    for dc in (-1, 1):
        s[(dc, 0)] = -2.0 * c0 * cx
        s[(2 * dc, 0)] = cx * cx
    for dr in (-1, 1):
        s[(0, dr)] = -2.0 * c0 * cy
        s[(0, 2 * dr)] = cy * cy
    for dc in (-1, 1):
        for dr in (-1, 1):
            s[(dc, dr)] = 2.0 * cx * cy
    return s


def solve(data: np.ndarray, difference: np.ndarray, dx: float, dy: float, mode: str,
          decay_length: float) -> np.ndarray:
    """The Height (order 1) or Slope (order 2) field."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    field = band(data, difference)
    d, _ = distances(data, dx, dy)
    unk = unknowns(data, d, REACH_DECAYS * decay_length)
    if not unk.any():
        return field
    order = 2 if mode == "slope" else 1
    st = _stencil(order, dx, dy, 1.0 / (decay_length * decay_length))
    h, w = data.shape
    rows, cols = np.nonzero(unk)
    index = np.full((h, w), -1, np.int64)
    index[rows, cols] = np.arange(len(rows))
    fixed = np.where(unk, 0.0, field.astype(np.float64))
    ai, aj, av = [], [], []
    rhs = np.zeros(len(rows))
    for (dc, dr), weight in st.items():
        r2, c2 = rows + dr, cols + dc  # unknowns are 3 posts off the border: in range
        j = index[r2, c2]
        m = j >= 0
        ai.append(np.arange(len(rows))[m])
        aj.append(j[m])
        av.append(np.full(int(m.sum()), weight))
        rhs -= weight * fixed[r2, c2]
    a = sp.csr_matrix((np.concatenate(av), (np.concatenate(ai), np.concatenate(aj))),
                      shape=(len(rows), len(rows)))
    x = spla.spsolve(a.tocsc(), rhs)
    out = field.copy()
    out[rows, cols] = x.astype(np.float32)
    return out


def cubic_weight(x: np.ndarray) -> np.ndarray:
    """The cubic convolution kernel with a = -0.5 (CubicWeight, src/raster/resample.cpp:20)."""
    a = -0.5
    x = np.abs(x)
    near = ((a + 2.0) * x - (a + 3.0)) * x * x + 1.0
    far = ((a * x - 5.0 * a) * x + 8.0 * a) * x - 4.0 * a
    return np.where(x <= 1.0, near, np.where(x < 2.0, far, 0.0))


def at(field: np.ndarray, lattice: tuple, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """SeamField::At (seam_field.cpp:644): the field between posts by Catmull-Rom over the 4 x 4
    posts around (x, y), 0 off the lattice, taps of zero weight skipped, summed in double and
    rounded to float. `lattice` is the GDAL transform of a north-up lattice."""
    x0, pw, _, y0, _, ph = lattice
    h, w = field.shape
    if not field.any():
        return np.zeros(np.shape(x))
    det = pw * ph
    px = ((x - x0) * ph) / det
    py = ((y - y0) * pw) / det
    fx, fy = px - 0.5, py - 0.5
    left, top = np.floor(fx), np.floor(fy)
    ok = (left >= -2.0) & (top >= -2.0) & (left <= w) & (top <= h)
    total = np.zeros(np.shape(x))
    for j in range(-1, 3):
        wy = cubic_weight((fy - top) - j)
        for i in range(-1, 3):
            wx = cubic_weight((fx - left) - i)
            c = np.where(ok, left + i, -1).astype(np.int64)
            r = np.where(ok, top + j, -1).astype(np.int64)
            inside = ok & (c >= 0) & (r >= 0) & (c < w) & (r < h)
            post = np.where(inside, field[np.clip(r, 0, h - 1), np.clip(c, 0, w - 1)], 0.0)
            weight = wx * wy
            total = total + np.where(weight == 0.0, 0.0, weight * post.astype(np.float64))
    return np.where(ok, total.astype(np.float32).astype(np.float64), 0.0)


def fill(field: np.ndarray, lattice: tuple, later: np.ndarray, grid, heights: np.ndarray):
    """SourceChain::FillGridGaps (src/sources/source_chain.cpp:167-192) on a north-up grid:
    cells of `heights` that are NaN take `later` plus the field at their centers (unchanged
    where the field reads 0; NaN where `later` is)."""
    rows, cols = np.nonzero(np.isnan(heights) & ~np.isnan(later))
    x = grid.x0 + (cols + 0.5) * grid.pixel
    y = grid.y0 + (rows + 0.5) * -grid.pixel
    correction = at(field, lattice, x, y)
    value = later[rows, cols]
    out = heights.copy()
    out[rows, cols] = np.where(correction == 0.0, value,
                               (value.astype(np.float64) + correction).astype(np.float32))
    return out


def chain(patches: list, windows: list, grid, mode: str, width: float = 50.0,
          decay_length: float = 50.0) -> np.ndarray:
    """SourceChain::FillSamples (src/sources/source_chain.cpp:154-192) of raster patches on
    windows (col0, row0, width, height) of `grid`: each later patch fills the cells the chain
    before it leaves without data, plus the seam of its link, whose lattice is the window of the
    patch before it padded by ceil(reach / spacing) + 3 posts (SourceChain::Seam, SeamLattice,
    source_chain.cpp:94-152)."""
    reach = width if mode == "feather" else REACH_DECAYS * decay_length
    pad = math.ceil(reach / grid.pixel) + 3
    h, w = grid.height, grid.width
    heights = np.full((h, w), np.nan, np.float32)

    def place(k):
        out = np.full((h, w), np.nan, np.float32)
        c0, r0, pw, ph = windows[k]
        out[r0:r0 + ph, c0:c0 + pw] = patches[k]
        return out

    heights[:] = place(0)
    for k in range(1, len(patches)):
        later = place(k)
        c0, r0, pw, ph = windows[k - 1]
        lc0, lr0, lw, lh = c0 - pad, r0 - pad, pw + 2 * pad, ph + 2 * pad
        data = np.zeros((lh, lw), np.uint8)
        diff = np.full((lh, lw), np.nan, np.float32)
        rows = np.arange(lr0, lr0 + lh)
        cols = np.arange(lc0, lc0 + lw)
        ri = (rows >= 0) & (rows < h)
        ci = (cols >= 0) & (cols < w)
        a = heights[np.ix_(rows[ri], cols[ci])]
        b = later[np.ix_(rows[ri], cols[ci])]
        has = np.isfinite(a)
        sub = data[np.ix_(ri, ci)]
        sub[:] = has
        data[np.ix_(ri, ci)] = sub
        both = has & np.isfinite(b)
        d = np.where(both, (a.astype(np.float64) - b).astype(np.float32), np.float32(np.nan))
        diff[np.ix_(ri, ci)] = d
        if mode == "feather":
            field = feather(data, diff, grid.pixel, grid.pixel, width)
        else:
            field = solve(data, diff, grid.pixel, grid.pixel, mode, decay_length)
        lattice = (grid.x0 + lc0 * grid.pixel, grid.pixel, 0.0, grid.y0 - lr0 * grid.pixel, 0.0,
                   -grid.pixel)
        heights = fill(field, lattice, later, grid, heights)
    return heights
