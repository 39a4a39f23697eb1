"""CPU restatement of the demo renderer's recording path -- TEST INFRASTRUCTURE ONLY.

Checks the library's headless renderer (arp_sim_render_rgb24).  It restates,
in numpy float32 operation by operation:

  * examples/test_mods/renderer.rs:40-68    vertex shader: density colour ramp,
                                            view matrix (:338-349), clip w
  * examples/test_mods/renderer.rs:90-128   fragment shader: point-sprite
                                            coordinate, disc test, poly6 alpha,
                                            sphere lighting
  * examples/test_mods/renderer.rs:250-272  blend and depth state of the two modes
  * examples/test_mods/renderer.rs:305-334  viewport, sprite size, clear colour

with the rasterisation rules the library states (fragments at pixel centres,
the sprite square half-open, 8-bit rounding after every blend) and draws the
sprites one at a time in draw order: boundary particles, then mobile
particles, each in caller order.

Parity of this restatement with the reference is unpinned: the reference
draws through OpenGL, which is unavailable on these machines, and GL leaves
point rasterisation and blend rounding to the implementation.
"""
import ctypes
import ctypes.util

import numpy as np

f32 = np.float32

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.cosf.restype = ctypes.c_float
_libm.cosf.argtypes = [ctypes.c_float]
_libm.sinf.restype = ctypes.c_float
_libm.sinf.argtypes = [ctypes.c_float]


def _to8(v):
    v = np.minimum(np.maximum(v, f32(0.0)), f32(1.0))
    return np.floor(v * f32(255.0) + f32(0.5)).astype(np.uint8)


def _from8(q):
    return q.astype(f32) / f32(255.0)


def render(boundary, particles, view, style, width, height, kconst):
    """RGB frame (height, width, 3), row 0 at the bottom.  `boundary` and
    `particles` are Particle records; `kconst` the poly6 constant of the
    fragment shader (normalization_constant(3, 3))."""
    recs = np.concatenate([boundary, particles])
    pos = recs["pos"].astype(f32)
    den = recs["den"].astype(f32)
    mat = recs["mat"].astype(np.int64)
    colors = np.asarray(style["colors"], f32).reshape(-1, 12)
    d0 = np.asarray(style["densities"], f32)
    s2 = min(width, height)
    vx0, vy0 = f32((width - s2) // 2), f32((height - s2) // 2)
    S = f32(s2) * f32(style["render_h"])
    ang = f32(view.get("angle", 0.0))
    ca, sa = f32(_libm.cosf(float(ang))), f32(_libm.sinf(float(ang)))
    tx = -f32(view.get("pos", (0.0, 0.0))[0])
    ty = f32(view.get("pos", (0.0, 0.0))[1])
    tz = -f32(view.get("scale", 1.0)) + f32(1.0)
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    x2 = (ca * x + (-sa) * z) + tx
    y2 = y + ty
    z2 = (sa * x + ca * z) + tz
    w = z2 + f32(1.0)
    with np.errstate(all="ignore"):
        ok = np.isfinite(pos[:, :3]).all(axis=1) & (w > 0) & (x2 >= -w) & (x2 <= w) & (y2 >= -w) & (y2 <= w) \
            & (z2 >= -w) & (z2 <= w) & (mat < len(colors))
        xn, yn, zn = x2 / w, y2 / w, z2 / w
        half = f32(0.5) * f32(s2)
        xw = (xn + f32(1.0)) * half + vx0
        yw = (yn + f32(1.0)) * half + vy0
        zw = (zn + f32(1.0)) * f32(0.5)
        m = np.minimum(mat, len(colors) - 1)
        dd = (den - d0[m]) / d0[m]
        base = colors[m, 0:4]
        other = np.where((dd < 0)[:, None], colors[m, 4:8], colors[m, 8:12])
        t = np.where(dd < 0, (-dd) / f32(5.0), dd / f32(5.0))
        col = base * (f32(1.0) - t)[:, None] + other * t[:, None]
        col[:, 3] = np.minimum(f32(1.0), col[:, 3])
    col[~ok, 3] = 0.0
    hs = f32(0.5) * S
    reach = np.minimum(f32(0.5) * S, S / (f32(4.0) * w)) + f32(1.0)

    def coverage(k):
        i0 = max(0, int(np.floor(xw[k] - reach[k])))
        i1 = min(width - 1, int(np.ceil(xw[k] + reach[k])))
        j0 = max(0, int(np.floor(yw[k] - reach[k])))
        j1 = min(height - 1, int(np.ceil(yw[k] + reach[k])))
        if i1 < i0 or j1 < j0:
            return None
        fx = (np.arange(i0, i1 + 1, dtype=f32) + f32(0.5))[None, :]
        fy = (np.arange(j0, j1 + 1, dtype=f32) + f32(0.5))[:, None]
        inside = (fx >= xw[k] - hs) & (fx < xw[k] + hs) & (fy >= yw[k] - hs) & (fy < yw[k] + hs)
        s = f32(0.5) + (fx - xw[k]) / S
        tt = f32(0.5) - (fy - yw[k]) / S
        px = (s - f32(0.5)) * f32(2.0)
        py = -((tt - f32(0.5)) * f32(2.0))
        dx = (px * f32(2.0)) * w[k]
        dy = (py * f32(2.0)) * w[k]
        dx, dy = np.broadcast_arrays(dx, dy)
        r2 = dx * dx + dy * dy
        return (slice(j0, j1 + 1), slice(i0, i1 + 1)), inside & (r2 <= f32(1.0)), dx, dy, r2

    if not style.get("lighting", False):
        q = np.zeros((height, width, 4), np.uint8)
        q[..., :3] = 255
        for k in range(len(recs)):
            if col[k, 3] == 0.0:
                continue
            cov = coverage(k)
            if cov is None:
                continue
            sl, mask, dx, dy, r2 = cov
            if not mask.any():
                continue
            diff = f32(1.0) - r2
            wk = ((f32(kconst) * diff) * diff) * diff
            sa_ = col[k, 3] * (wk / f32(kconst))
            tile = q[sl]
            da = _from8(tile[..., 3])
            new = np.empty_like(tile)
            for c in range(3):
                new[..., c] = _to8(col[k, c] * (f32(1.0) - da) + _from8(tile[..., c]) * (f32(1.0) - sa_))
            new[..., 3] = _to8(sa_ * da + da * sa_)
            tile[mask] = new[mask]
        return q[..., :3]
    # lighting: nearest sprite per pixel (LESS, first drawn on ties), then sphere shading
    zbest = np.full((height, width), np.inf, f32)
    who = np.full((height, width), -1, np.int64)
    for k in range(len(recs)):
        if col[k, 3] == 0.0 or not (zw[k] < 1.0 and zw[k] >= 0.0):
            continue
        cov = coverage(k)
        if cov is None:
            continue
        sl, mask, dx, dy, r2 = cov
        better = mask & (zw[k] < zbest[sl])
        zbest[sl][better] = zw[k]
        who[sl][better] = k
    out = np.full((height, width, 3), 255, np.uint8)
    rh = f32(style["render_h"])
    lp = np.asarray(style.get("light_pos", (-3, 3, -3)), f32)
    lc = np.asarray(style.get("light_color", (1, 1, 1)), f32)
    amb, dif, spc = f32(style.get("ambient", 1.0)), f32(style.get("diffuse", 10.0)), f32(style.get("specular", 0.0))
    for j, i in zip(*np.nonzero(who >= 0)):
        k = who[j, i]
        fx, fy = f32(i) + f32(0.5), f32(j) + f32(0.5)
        s = f32(0.5) + (fx - xw[k]) / S
        tt = f32(0.5) - (fy - yw[k]) / S
        dx = ((s - f32(0.5)) * f32(2.0) * f32(2.0)) * w[k]
        dy = ((-((tt - f32(0.5)) * f32(2.0))) * f32(2.0)) * w[k]
        nz = -np.sqrt(f32(1.0) - dx * dx - dy * dy)
        sp = np.array([x2[k] + rh * dx, y2[k] + rh * dy, z2[k] + rh * nz], f32)
        lv = lp - sp
        ll = f32(1.0) / np.sqrt(np.dot(lv, lv))
        lv = lv * (ll * ll * ll)
        nrm = np.array([dx, dy, nz], f32)
        diffuse = np.dot(lv, nrm)
        rz = lv[2] - f32(2.0) * np.dot(nrm, lv) * nz
        spec = max(f32(20.0) * rz, f32(0.0))
        spec = spec * spec * spec
        out[j, i] = _to8(col[k, :3] * amb + diffuse * dif * lc + lc * spec * spc)
    return out
