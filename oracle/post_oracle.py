"""ORACLE -- test infrastructure only.  Numpy restatement (float64) of the reference's
post-processing passes, for the parity tests of s2_temporal_accumulate and s2_tonemap:

* temporal accumulation: src/Shaders/kernels/svgf/temporal_accumulation.slang:34-129 (debug modes
  left out), with the defaults of src/App/Denoiser.cpp:24-26 and Denoiser.hpp:54-58;
* tonemapping: src/Shaders/kernels/tonemap.slang:30-192 (maxReduce + main), the operators in
  TonemapMode order (compat/tonemap.h), rgbToSrgb / viridisQuintic / luminance of
  src/Shaders/compat/common.h:51, 88-104.
"""
from __future__ import annotations

import numpy as np

REPROJECT, CHECK_NORMAL, CHECK_DEPTH, DEMODULATE_ALBEDO, SHADOW_HYSTERESIS = 1, 2, 4, 8, 16
LUM = np.array([0.2126, 0.7152, 0.0722])


def luminance(c):
    return np.asarray(c, np.float64)[..., :3] @ LUM


def unpack_normal(p):
    """Octahedral SNORM16 decode of the visibility AOV's normal (unpackNormal; the octahedral wrap
    of the lower hemisphere, then normalisation)."""
    p = int(p) & 0xFFFFFFFF
    sx = (p & 0xFFFF) - (1 << 16 if p & 0x8000 else 0)
    sy = (p >> 16) - (1 << 16 if p & 0x80000000 else 0)
    x, y = max(sx / 32767.0, -1.0), max(sy / 32767.0, -1.0)
    z = 1.0 - (abs(x) + abs(y))
    if z < 0:
        x, y = (1.0 - abs(y)) * (1.0 if x >= 0 else -1.0), (1.0 - abs(x)) * (1.0 if y >= 0 else -1.0)
    v = np.array([x, y, z])
    return v / np.linalg.norm(v)


def temporal_accumulate(radiance, albedo, vis, depth, prev_uv, prev, flags, history_limit=0, shadow_offset=0.1,
                        shadow_scale=1.0, instance_map=None):
    """One frame.  Images are (H, W, c) arrays of the view (image_min = 0); `prev` is None (no
    history) or a dict with color (H, W, 4), moments (H, W, 2), vis (H, W, 2), depth (H, W, 4).
    Returns (color, moments)."""
    H, W = radiance.shape[:2]
    color = np.zeros((H, W, 4))
    moments = np.zeros((H, W, 2))
    cos_limit = np.cos(np.degrees(2.0))  # cos(degrees(2)) as written in the shader
    for y in range(H):
        for x in range(W):
            cprev = np.zeros(4)
            mprev = np.zeros(2)
            sw = 0.0
            if prev is not None:
                if flags & REPROJECT:
                    inst = int(vis[y, x, 0]) & 0xFFFF
                    if inst != 0xFFFF:
                        # the tap position in single precision, as the shader computes it (its
                        # truncation decides which taps are read)
                        px = float(np.float32(np.float32(prev_uv[y, x, 0]) * np.float32(W)) - np.float32(0.5))
                        py = float(np.float32(np.float32(prev_uv[y, x, 1]) * np.float32(H)) - np.float32(0.5))
                        p0x, p0y = int(px), int(py)  # int2(): truncation
                        wx, wy = px - np.floor(px), py - np.floor(py)  # frac()
                        n = unpack_normal(vis[y, x, 1])
                        mapped = instance_map[inst] if instance_map is not None else inst
                        for yy in (0, 1):
                            for xx in (0, 1):
                                qx, qy = p0x + xx, p0y + yy
                                if not (0 <= qx < W and 0 <= qy < H):
                                    continue
                                pv = prev["vis"][qy, qx]
                                if mapped != (int(pv[0]) & 0xFFFF):
                                    continue
                                if (flags & CHECK_NORMAL) and np.dot(n, unpack_normal(pv[1])) < cos_limit:
                                    continue
                                if (flags & CHECK_DEPTH) and abs(depth[y, x, 1] - prev["depth"][qy, qx, 0]) >= \
                                        2 * np.hypot(depth[y, x, 2], depth[y, x, 3]):
                                    continue
                                c = prev["color"][qy, qx]
                                if c[3] <= 0 or not np.all(np.isfinite(c)):
                                    continue
                                wc = (1 - wx if xx == 0 else wx) * (1 - wy if yy == 0 else wy)
                                cprev = cprev + c * wc
                                mprev = mprev + prev["moments"][qy, qx] * wc
                                sw += wc
                else:
                    cprev = prev["color"][y, x].astype(np.float64)
                    if not np.all(np.isfinite(cprev[:3])):
                        cprev = np.zeros(4)
                    else:
                        mprev = prev["moments"][y, x].astype(np.float64)
                    sw = 1.0
            cur = radiance[y, x].astype(np.float64).copy()
            if flags & DEMODULATE_ALBEDO:
                cur[:3] = cur[:3] / (1e-2 + albedo[y, x, :3])
            if not np.all(np.isfinite(cur[:3])):
                cur = np.zeros(4)
            if not np.all(np.isfinite(mprev)):
                mprev = np.zeros(2)
            l = float(cur[:3] @ LUM)
            if sw > 0 and cprev[3] > 0:
                cprev = cprev / sw
                mprev = mprev / sw
                n = cprev[3] + cur[3]
                if history_limit > 0 and n > history_limit:
                    n = history_limit
                alpha = min(max(cur[3] / n, 0.0), 1.0)
                if flags & SHADOW_HYSTERESIS:
                    lp = float(cprev[:3] @ LUM)
                    r = 0.0 if l + lp == 0 else (lp - l) / (l + lp)
                    al = min(max(r - shadow_offset, 0.0), 1.0) ** 2 * shadow_scale
                    alpha = 1 - (1 - alpha) * min(max(1 - al, 0.0), 1.0)
                color[y, x, :3] = cprev[:3] + (cur[:3] - cprev[:3]) * alpha
                color[y, x, 3] = n
                moments[y, x] = mprev + (np.array([l, l * l]) - mprev) * alpha
            else:
                color[y, x] = cur
                moments[y, x] = (l, l * l)
    return color, moments


# ------------------------------------------------------------------------------ tonemapping
def rgb_to_srgb_reference(c):
    """rgbToSrgb of compat/common.h:88-93 as written: pow(1.055 x, 1/2.4) - 0.055 (not sRGB)."""
    c = np.asarray(c, np.float64)
    return np.where(c <= 0.0031308, c * 12.92, np.power(np.maximum(c * 1.055, 0), 1 / 2.4) - 0.055)


def rgb_to_srgb(c):
    """The standard sRGB encoding: 1.055 x^(1/2.4) - 0.055 above 0.0031308."""
    c = np.asarray(c, np.float64)
    return np.where(c <= 0.0031308, c * 12.92, 1.055 * np.power(np.maximum(c, 0), 1 / 2.4) - 0.055)


def viridis(x):
    """viridisQuintic (compat/common.h:96-104)."""
    x = np.asarray(x, np.float64)[..., None]
    p = np.concatenate([np.ones_like(x), x, x ** 2, x ** 3, x ** 4, x ** 5], -1)
    k = np.array([[0.280268003, -0.143510503, 2.225793877, -14.815088879, 25.212752309, -11.772589584],
                  [-0.002117546, 1.617109353, -1.909305070, 2.701152864, -1.685288385, 0.178738871],
                  [0.300805501, 2.614650302, -12.019139090, 28.933559110, -33.491294770, 13.762053843]])
    return p @ k.T


def _hable(x):
    A, B, C, D, E, F = 0.15, 0.50, 0.10, 0.20, 0.02, 0.30
    return ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - E / F


def tonemap(img, mode, exposure=0.0, gamma=False, gamma_reference=False, albedo=None):
    """tonemap.slang maxReduce + main for an (H, W, 4) image; returns (H, W, 4) with alpha 1."""
    img = np.asarray(img, np.float64)[..., :3]
    # maxReduce: per-channel and luminance maxima of (albedo x) input, quantized to 1/16384
    v = img * albedo[..., :3] if albedo is not None else img.copy()
    w = v @ LUM
    ok = np.all(np.isfinite(v), -1) & np.isfinite(w) & (w > 0)
    q = lambda a: np.floor(np.clip(a * 16384.0, 0, 4294967295.0)) if a.size else np.zeros(0)
    mx = np.zeros(4)
    if ok.any():
        mx[:3] = q(v[ok]).max(0)
        mx[3] = q(w[ok]).max()
    mx = mx / 16384.0
    c = img * (1e-2 + albedo[..., :3]) if albedo is not None else img.copy()
    c = c * 2.0 ** exposure
    maxc, maxl = mx[:3], mx[3]
    with np.errstate(divide="ignore", invalid="ignore"):
        if mode == 1:    # Reinhard
            l = (c @ LUM)[..., None]
            tc = c / (1 + c)
            cl = c / (1 + l)
            c = cl + (tc - cl) * tc
        elif mode == 2:  # Reinhard extended
            m = np.where(maxc == 0, 1.0, maxc)
            c = c / (1 + c) * (1 + c / m ** 2)
        elif mode == 3:  # Reinhard luminance
            l = (c @ LUM)[..., None]
            c = c * ((l / (1 + l)) / l)
        elif mode == 4:  # Reinhard luminance extended
            l = (c @ LUM)[..., None]
            m = 1.0 if maxl == 0 else maxl
            c = c * (((l / (1 + l)) * (1 + l / m ** 2)) / l)
        elif mode == 5:  # Uncharted 2
            c = _hable(c) / _hable(1.0 if maxl == 0 else maxl)
        elif mode == 6:  # filmic
            x = np.maximum(0, c - 0.004)
            c = (x * (6.2 * x + 0.5)) / (x * (6.2 * x + 1.7) + 0.06)
        elif mode == 7:  # ACES fitted
            mi = np.array([[0.59719, 0.35458, 0.04823], [0.07600, 0.90834, 0.01566], [0.02840, 0.13383, 0.83777]])
            mo = np.array([[1.60475, -0.53108, -0.07367], [-0.10208, 1.10813, -0.00605], [-0.00327, -0.07276, 1.07602]])
            v2 = c @ mi.T
            v2 = (v2 * (v2 + 0.0245786) - 0.000090537) / (v2 * (0.983729 * v2 + 0.4329510) + 0.238081)
            c = np.clip(v2 @ mo.T, 0, 1)
        elif mode == 8:  # ACES approximation
            x = c * 0.6
            c = np.clip((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0, 1)
        elif mode == 9:  # viridis of the luminance
            c = viridis(np.clip(c @ LUM, 0, 1))
        elif mode == 10:  # viridis of the luminance over the maximum
            c = viridis(np.clip((c @ LUM) / (1.0 if maxl == 0 else maxl), 0, 1))
    if gamma_reference:
        c = rgb_to_srgb_reference(c)
    elif gamma:
        c = rgb_to_srgb(c)
    return np.concatenate([c, np.ones(c.shape[:-1] + (1,))], -1)


# ------------------------------------------------------------------------------ SVGF
def svgf_variance(color, moments, vis, depth, flags, history_limit=0, boost=4.0, instance_map=None):
    """estimate_variance.slang main (:26-74): (H, W, 4) of (rgb, variance)."""
    H, W = color.shape[:2]
    out = np.zeros((H, W, 4))
    for y in range(H):
        for x in range(W):
            c = color[y, x].astype(np.float64).copy()
            m = moments[y, x].astype(np.float64).copy()
            inst = int(vis[y, x, 0]) & 0xFFFF
            if inst == 0xFFFF or c[3] >= history_limit:
                out[y, x] = (*c[:3], abs(m[1] - m[0] ** 2))
                continue
            n = unpack_normal(vis[y, x, 1])
            mapped = instance_map[inst] if instance_map is not None else inst
            d = depth[y, x]
            sw = 1.0
            r = 2 if c[3] > 1 else 3
            for yy in range(-r, r + 1):
                for xx in range(-r, r + 1):
                    if xx == 0 and yy == 0:
                        continue
                    px, py = x + xx, y + yy
                    if not (0 <= px < W and 0 <= py < H) or (int(vis[py, px, 0]) & 0xFFFF) != mapped:
                        continue
                    wz = abs(depth[py, px, 0] - d[0]) / (np.hypot(d[2] * xx, d[3] * yy) + 1e-2) if flags & CHECK_DEPTH else 0.0
                    wn = min(max(float(np.dot(unpack_normal(vis[py, px, 1]), n)), 0.0), 1.0) ** 128 if flags & CHECK_NORMAL else 1.0
                    w = np.exp(-wz) * wn
                    if not np.isfinite(w):
                        continue
                    m = m + moments[py, px] * w
                    c[:3] = c[:3] + color[py, px, :3] * w
                    sw += w
            m, c[:3] = m / sw, c[:3] / sw
            v = abs(m[1] - m[0] ** 2)
            if boost > 0:
                v *= max(1.0, boost / (1 + c[3]))
            out[y, x] = (*c[:3], v)
    return out


def _svgf_taps(kernel, it, st):
    if kernel == 4:
        kernel = 1 if st == 1 else 3
    if kernel == 5:
        kernel = 2 if st == 1 else 3
    if kernel == 0:  # atrous (atrous.slang:136-170)
        k1 = [1.0, 2 / 3, 1 / 6]
        return [(xx * st, yy * st, k1[abs(xx) + abs(yy)] if xx == 0 or yy == 0 else k1[abs(xx)] * k1[abs(yy)])
                for yy in range(-2, 3) for xx in range(-2, 3) if xx or yy]
    if kernel == 3:  # subsampled (:84-118)
        pair = [(-2 * st, 0, 1.0), (2 * st, 0, 1.0)] if it % 2 == 0 else [(0, -2 * st, 1.0), (0, 2 * st, 1.0)]
        return pair + [(-st, st, 1.0), (st, st, 1.0), (-st, -st, 1.0), (st, -st, 1.0)]
    r = 2 if kernel == 2 else 1
    return [(xx * st, yy * st, 1.0) for yy in range(-r, r + 1) for xx in range(-r, r + 1) if xx or yy]


def svgf_atrous(img, vis, depth, it, kernel, flags, sigma_boost=3.0):
    """One atrous.slang pass (:180-227), step 2^it."""
    H, W = img.shape[:2]
    st = 1 << it
    out = np.zeros((H, W, 4))
    for y in range(H):
        for x in range(W):
            c = img[y, x].astype(np.float64)
            s = c[3] / 16.0
            for yy in (-1, 0, 1):
                for xx in (-1, 0, 1):
                    if (xx or yy) and 0 <= x + xx < W and 0 <= y + yy < H:
                        s += img[y + yy, x + xx, 3] * (1 / 8 if xx == 0 or yy == 0 else 1 / 16)
            sigma = np.sqrt(max(s, 0.0)) * sigma_boost
            lc = float(c[:3] @ LUM)
            nc = unpack_normal(vis[y, x, 1])
            zc, dz = depth[y, x, 0], depth[y, x, 2:4]
            acc, sw = c.copy(), 1.0
            if np.isfinite(zc):
                for ox, oy, kw in _svgf_taps(kernel, it, st):
                    px, py = x + ox, y + oy
                    if not (0 <= px < W and 0 <= py < H):
                        continue
                    cp = img[py, px].astype(np.float64)
                    wl = abs(float(cp[:3] @ LUM) - lc) / max(sigma, 1e-10)
                    wz = abs(depth[py, px, 0] - zc) / (np.hypot(dz[0] * ox * st, dz[1] * oy * st) + 1e-2) if flags & CHECK_DEPTH else 0.0
                    wn = max(0.0, float(np.dot(unpack_normal(vis[py, px, 1]), nc))) ** 256 if flags & CHECK_NORMAL else 1.0
                    w = np.exp(-wl * wl - wz) * kw * wn
                    if not np.isfinite(w):
                        continue
                    acc = acc + cp * np.array([w, w, w, w * w])
                    sw += w
            out[y, x] = acc * np.array([1 / sw, 1 / sw, 1 / sw, 1 / sw ** 2])
    return out
