"""ORACLE -- test infrastructure only.  Numpy restatement (float64) of the reference's texture repack
of a glTF metallic-roughness material, for the parity tests of s2_repack_metallic_roughness and for
CPU tests of the glTF loader (which take it as the loader's `repack` argument):

* from_gltf_pbr, src/Shaders/kernels/convert_material.slang:33-69: per texel, PackedMaterialData
  of the base colour, metallic-roughness (metallic b, roughness g) and emission textures, with the
  fixed values 1 for specular, sheen, anisotropic, subsurface, clearcoat, clearcoat gloss,
  transmission and eta; the base colour's alpha as the alpha mask and InterlockedMin of the 8-bit
  alpha of texels with alpha < 1;
* the setters' quantisation floor(saturate(v) * 255 + 0.5) (src/Shaders/compat/material_data.h:
  51-73), setEmission's normalisation by the largest channel, and PackedMaterialData::Store's
  byte / 255 (src/Shaders/common/material.hlsli:113-118);
* the sRGB decode of the base colour and emission textures (their sRGB formats,
  load_gltf.cpp:46-48) as srgbToRgb, src/Shaders/compat/common.h:81-86.

Inputs are RGBA8 uint8 arrays (None = absent, read as 1); every step is float64, as in the device
kernel, so the two agree exactly for 8-bit inputs.
"""
from __future__ import annotations

import numpy as np


def srgb_to_linear(c):
    """srgbToRgb (compat/common.h:81-86)."""
    c = np.asarray(c, np.float64)
    return np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)


def _q(v):
    """setX's 8-bit quantisation followed by Store's byte / 255, as float32."""
    b = np.floor(np.clip(np.asarray(v, np.float64), 0.0, 1.0) * 255.0 + 0.5)
    return b.astype(np.float32) / np.float32(255.0)


def repack_metallic_roughness(base=None, metallic_roughness=None, emission=None):
    """-> (four packed images float32 (h, w, 4), base alpha float32 (h, w) or None, min alpha)."""
    src = [None if t is None else np.asarray(t, np.uint8) for t in (base, metallic_roughness, emission)]
    ref = next(t for t in src if t is not None)
    h, w = ref.shape[:2]
    full = np.full((h, w, 4), 255, np.uint8)
    d8, m8, e8 = (t if t is not None else full for t in src)
    lin = srgb_to_linear(np.arange(256) / 255.0)
    d = lin[d8[..., :3]]
    ones = np.ones((h, w), np.float32)
    img0 = np.concatenate([_q(d), ones[..., None]], -1)
    e = lin[e8[..., :3]]
    emax = e.max(-1, keepdims=True)
    en = np.where(emax > 0, e / np.where(emax > 0, emax, 1.0), 0.0)       # 0/0 saturates to 0
    img1 = np.concatenate([_q(en), ones[..., None]], -1)
    img2 = np.stack([m8[..., 2].astype(np.float32) / np.float32(255.0),
                     m8[..., 1].astype(np.float32) / np.float32(255.0), ones, ones], -1)
    img3 = np.ones((h, w, 4), np.float32)
    alpha, min_alpha = None, 255
    if src[0] is not None:
        a8 = src[0][..., 3]
        alpha = a8.astype(np.float32) / np.float32(255.0)
        below = a8 < 255
        if below.any():
            min_alpha = int(a8[below].min())
    return [img0, img1, img2, img3], alpha, min_alpha
