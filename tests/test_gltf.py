"""glTF ingest (stratum2_b200/gltf.py): a document written here (two meshes under a node
hierarchy, materials with factors, extensions and PNG textures, a camera) loads the same from
.gltf with data URIs and from .glb; transforms, materials, the per-texel texture repack
(from_gltf_pbr, convert_material.slang:33-69, through the oracle's restatement standing in for the
GPU repack) and the PNG and JPEG decoders are checked against direct computations.  CPU only; the
GPU repack and a glTF render are compared with the oracle in tests/test_gltf_gpu.py."""
import base64
import io
import json
import struct
import sys
import zlib
from pathlib import Path

import numpy as np
import pytest

from stratum2_b200 import _abi
from stratum2_b200.gltf import decode_image_rgba8, decode_png, load_gltf
from stratum2_b200.scene import Material, rotation_from_quaternion

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
from gltf_oracle import repack_metallic_roughness, srgb_to_linear  # noqa: E402

REPACK = repack_metallic_roughness


def png_encode(px: np.ndarray, filters=(0, 1, 2, 3, 4)) -> bytes:
    """RGBA8 PNG with the given filter types cycled over the rows (encoder for the tests)."""
    h, w, ch = px.shape
    rows, prev = [], np.zeros(w * ch, np.int32)
    for y in range(h):
        line = px[y].reshape(-1).astype(np.int32)
        f = filters[y % len(filters)]
        left = np.concatenate([np.zeros(ch, np.int32), line[:-ch]])
        upleft = np.concatenate([np.zeros(ch, np.int32), prev[:-ch]])
        if f == 0:
            enc = line
        elif f == 1:
            enc = line - left
        elif f == 2:
            enc = line - prev
        elif f == 3:
            enc = line - ((left + prev) >> 1)
        else:
            p = left + prev - upleft
            pa, pb, pc = np.abs(p - left), np.abs(p - prev), np.abs(p - upleft)
            pred = np.where((pa <= pb) & (pa <= pc), left, np.where(pb <= pc, prev, upleft))
            enc = line - pred
        rows.append(bytes([f]) + (enc & 0xFF).astype(np.uint8).tobytes())
        prev = line

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    ctype = {1: 0, 3: 2, 4: 6}[ch]
    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, ctype, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(b"".join(rows))) + chunk(b"IEND", b""))


@pytest.mark.parametrize("ch", [1, 3, 4])
def test_png_decoder_all_filters(ch):
    rng = np.random.default_rng(ch)
    px = rng.integers(0, 256, (7, 9, ch), dtype=np.uint8)
    out = decode_png(png_encode(px))
    ref = np.full((7, 9, 4), 255, np.uint8)
    ref[..., :3] = px[..., :1] if ch == 1 else px[..., :3]
    if ch == 4:
        ref[..., 3] = px[..., 3]
    np.testing.assert_array_equal(np.round(out * 255).astype(np.uint8), ref)


def _document(rng):
    base_px = rng.integers(0, 256, (4, 4, 4), dtype=np.uint8)
    base_px[0, 0, 3] = 64  # an alpha below 1: the base colour's alpha becomes the mask
    mr_px = rng.integers(0, 256, (4, 4, 3), dtype=np.uint8)
    quad = np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], np.float32)
    quad_n = np.tile(np.array([[0, 1, 0]], np.float32), (4, 1))
    quad_uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    quad_i = np.array([0, 1, 2, 0, 2, 3], np.uint16)
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    blobs = [quad.tobytes(), quad_n.tobytes(), quad_uv.tobytes(), quad_i.tobytes() + b"\0\0", tri.tobytes()]
    offs = np.cumsum([0] + [len(b) for b in blobs])
    data = b"".join(blobs)
    views = [{"buffer": 0, "byteOffset": int(offs[k]), "byteLength": len(blobs[k])} for k in range(5)]
    views[3]["byteLength"] = len(quad_i.tobytes())
    acc = [
        {"bufferView": 0, "componentType": 5126, "count": 4, "type": "VEC3"},
        {"bufferView": 1, "componentType": 5126, "count": 4, "type": "VEC3"},
        {"bufferView": 2, "componentType": 5126, "count": 4, "type": "VEC2"},
        {"bufferView": 3, "componentType": 5123, "count": 6, "type": "SCALAR"},
        {"bufferView": 4, "componentType": 5126, "count": 3, "type": "VEC3"},
    ]
    uri = lambda b, kind: f"data:{kind};base64," + base64.b64encode(b).decode()
    doc = {
        "asset": {"version": "2.0"},
        "scene": 0,
        "scenes": [{"nodes": [0, 3]}],
        "nodes": [
            {"translation": [0.5, 1.0, -2.0], "rotation": [0.0, 0.38268343, 0.0, 0.92387953], "scale": [2, 2, 2],
             "children": [1, 2]},
            {"mesh": 0, "matrix": [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0.1, 0.2, 0.3, 1]},
            {"mesh": 1},
            {"camera": 0, "translation": [0, 5, 4], "rotation": [-0.3826834, 0.0, 0.0, 0.9238795]},
        ],
        "cameras": [{"type": "perspective", "perspective": {"yfov": 0.7, "znear": 0.01}}],
        "meshes": [
            {"primitives": [{"attributes": {"POSITION": 0, "NORMAL": 1, "TEXCOORD_0": 2}, "indices": 3, "material": 0}]},
            {"primitives": [{"attributes": {"POSITION": 4}, "material": 1}]},
        ],
        "materials": [
            {"pbrMetallicRoughness": {"baseColorFactor": [0.9, 0.8, 0.7, 1.0], "roughnessFactor": 0.6,
                                      "metallicFactor": 0.3, "baseColorTexture": {"index": 0},
                                      "metallicRoughnessTexture": {"index": 1}},
             "emissiveFactor": [0.5, 0.25, 0.0],
             "extensions": {"KHR_materials_emissive_strength": {"emissiveStrength": 4.0},
                            "KHR_materials_ior": {"ior": 1.33}}},
            {"pbrMetallicRoughness": {"baseColorFactor": [0.2, 0.4, 0.6, 1.0], "roughnessFactor": 0.25,
                                      "metallicFactor": 0.0},
             "extensions": {"KHR_materials_transmission": {"transmissionFactor": 0.5},
                            "KHR_materials_clearcoat": {"clearcoatFactor": 0.75},
                            "KHR_materials_specular": {"specularFactor": 0.4}}},
        ],
        "textures": [{"source": 0}, {"source": 1}],
        "images": [{"uri": uri(png_encode(base_px), "image/png")}, {"uri": uri(png_encode(mr_px), "image/png")}],
        "buffers": [{"byteLength": len(data), "uri": uri(data, "application/octet-stream")}],
        "bufferViews": views,
        "accessors": acc,
    }
    return doc, data, base_px, mr_px, quad, tri


def _write_glb(doc, data, path):
    d = json.loads(json.dumps(doc))
    d["buffers"] = [{"byteLength": len(data)}]
    js = json.dumps(d).encode()
    js += b" " * (-len(js) % 4)
    bin_ = data + b"\0" * (-len(data) % 4)
    body = struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(bin_), 0x004E4942) + bin_
    path.write_bytes(struct.pack("<III", 0x46546C67, 2, 12 + len(body)) + body)


def test_gltf_and_glb_load_the_same_scene(tmp_path):
    doc, data, base_px, mr_px, quad, tri = _document(np.random.default_rng(0))
    (tmp_path / "s.gltf").write_text(json.dumps(doc))
    _write_glb(doc, data, tmp_path / "s.glb")
    a, b = load_gltf(tmp_path / "s.gltf", repack=REPACK), load_gltf(tmp_path / "s.glb", repack=REPACK)
    assert a.instances == b.instances == 2
    assert bytes(a.scene.material_data) == bytes(b.scene.material_data)
    for x, y in zip(a.scene.vertex_buffers + a.scene.images + a.scene.transforms,
                    b.scene.vertex_buffers + b.scene.images + b.scene.transforms):
        np.testing.assert_array_equal(x, y)


def test_gltf_transforms_materials_and_repack(tmp_path):
    doc, data, base_px, mr_px, quad, tri = _document(np.random.default_rng(0))
    (tmp_path / "s.gltf").write_text(json.dumps(doc))
    g = load_gltf(tmp_path / "s.gltf", width=64, height=48, repack=REPACK)
    s = g.scene
    # parent TRS x child matrix; second mesh under the parent alone
    parent = np.eye(4)
    parent[:3, :3] = rotation_from_quaternion((0.0, 0.38268343, 0.0, 0.92387953)) @ np.diag([2, 2, 2])
    parent[:3, 3] = (0.5, 1.0, -2.0)
    child = np.eye(4)
    child[:3, 3] = (0.1, 0.2, 0.3)
    np.testing.assert_allclose(np.asarray(s.transforms[0]).reshape(3, 4), (parent @ child)[:3], atol=1e-6)
    np.testing.assert_allclose(np.asarray(s.transforms[1]).reshape(3, 4), parent[:3], atol=1e-6)
    # materials: makeMetallicRoughnessMaterial of the factors plus the extensions
    m0 = Material.metallic_roughness((0.9, 0.8, 0.7), 0.6, 0.3, emission=(2.0, 1.0, 0.0), eta=1.33)
    m1 = Material.metallic_roughness((0.2, 0.4, 0.6), 0.25, 0.0, transmission=0.5)
    m1.clearcoat, m1.specular = 0.75, 0.4
    assert s.materials[0].packed_words() == m0.packed_words()
    assert s.materials[1].packed_words() == m1.packed_words()
    assert s.materials[1].images == (_abi.NO_IMAGE,) * 4
    # texture repack: image 0 = sRGB-decoded base colour (+ specular 1), image 2 = metallic (B),
    # roughness (G), no emission or packed[3] images, alpha mask from the base colour's alpha
    im = s.materials[0].images
    assert im[1] == _abi.NO_IMAGE and im[3] == _abi.NO_IMAGE
    base_lin = srgb_to_linear(base_px[..., :3] / 255.0)
    np.testing.assert_allclose(s.images[im[0]][..., :3], np.floor(base_lin * 255 + 0.5) / 255, atol=1e-7)
    np.testing.assert_allclose(s.images[im[0]][..., 3], 1.0)
    np.testing.assert_allclose(s.images[im[2]][..., 0], mr_px[..., 2] / 255.0, atol=1e-7)
    np.testing.assert_allclose(s.images[im[2]][..., 1], mr_px[..., 1] / 255.0, atol=1e-7)
    mask = s.materials[0].alpha_mask
    assert mask != _abi.NO_IMAGE
    np.testing.assert_allclose(s.images[mask][..., 0], base_px[..., 3] / 255.0, atol=1e-7)
    # camera: a view at the camera node
    assert len(g.views) == 1
    np.testing.assert_allclose([g.views[0].camera_to_world[k] for k in (3, 7, 11)], (0, 5, 4), atol=1e-6)
    # looking down 45 degrees: the camera's -z axis
    np.testing.assert_allclose([-g.views[0].camera_to_world[k] for k in (2, 6, 10)], (0, -0.7071068, -0.7071068), atol=1e-5)


def test_repack_per_texel_packing():
    """The oracle's repack of every texel equals Material.packed_words (pinned to the reference's
    PackedMaterialData setters) of the texel's sRGB-decoded values."""
    rng = np.random.default_rng(3)
    base = rng.integers(0, 256, (3, 5, 4), dtype=np.uint8)
    emis = rng.integers(0, 256, (3, 5, 4), dtype=np.uint8)
    emis[0, 0, :3] = 0  # black emission: 0/0 saturates to 0
    imgs, _, _ = repack_metallic_roughness(base, None, emis)
    for y, x in ((0, 0), (2, 4), (1, 3)):
        m = Material(base_color=tuple(srgb_to_linear(base[y, x, :3] / 255.0)),
                     emission=tuple(srgb_to_linear(emis[y, x, :3] / 255.0)), specular=1.0, sheen=1.0)
        w, _ = m.packed_words()
        got0 = np.round(imgs[0][y, x] * 255).astype(int)
        got1 = np.round(imgs[1][y, x] * 255).astype(int)
        assert list(got0) == [(w[0] >> (8 * k)) & 0xFF for k in range(4)]
        assert list(got1) == [(w[1] >> (8 * k)) & 0xFF for k in range(4)]


def test_textured_material_needs_the_gpu_repack(tmp_path):
    doc, *_ = _document(np.random.default_rng(0))
    (tmp_path / "s.gltf").write_text(json.dumps(doc))
    with pytest.raises(ValueError, match="repacked on the GPU"):
        load_gltf(tmp_path / "s.gltf")


def _jpeg(px: np.ndarray, quality: int = 95) -> bytes:
    from PIL import Image
    buf = io.BytesIO()
    Image.fromarray(px).save(buf, format="JPEG", quality=quality, subsampling=0)
    return buf.getvalue()


def test_jpeg_and_png_decode_by_signature():
    yy, xx = np.mgrid[0:24, 0:40]
    px = np.stack([xx * 6, yy * 10, (xx + yy) * 4], -1).astype(np.uint8)  # smooth: small JPEG error
    j = decode_image_rgba8(_jpeg(px))
    assert j.shape == (24, 40, 4) and j.dtype == np.uint8 and (j[..., 3] == 255).all()
    assert np.abs(j[..., :3].astype(int) - px).max() <= 6
    rgba = np.concatenate([px, np.full((24, 40, 1), 200, np.uint8)], -1)
    np.testing.assert_array_equal(decode_image_rgba8(png_encode(rgba)), rgba)
    with pytest.raises(ValueError, match="unsupported image format"):
        decode_image_rgba8(b"GIF89a" + b"\0" * 32)


def test_gltf_with_a_jpeg_texture(tmp_path):
    """A JPEG base-colour texture goes through the same repack as a PNG one: the repack's input is
    the decoded RGBA8."""
    doc, data, base_px, *_ = _document(np.random.default_rng(0))
    smooth = np.repeat(np.repeat(base_px[:1, :1, :3], 4, 0), 4, 1)  # one colour: JPEG keeps it within a step
    doc["images"][0]["uri"] = "data:image/jpeg;base64," + base64.b64encode(_jpeg(smooth)).decode()
    (tmp_path / "s.gltf").write_text(json.dumps(doc))
    seen = []

    def spy(*a):
        seen.append(a)
        return REPACK(*a)

    g = load_gltf(tmp_path / "s.gltf", repack=spy)
    base_in = seen[0][0]
    assert base_in.shape == (4, 4, 4) and (base_in[..., 3] == 255).all()
    assert np.abs(base_in[..., :3].astype(int) - smooth).max() <= 2
    assert g.scene.materials[0].alpha_mask == _abi.NO_IMAGE  # JPEG has no alpha
