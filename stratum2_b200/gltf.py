"""glTF 2.0 ingest (.gltf with embedded or external buffers, and .glb) into a Scene, as the
reference's loader does it (src/App/loaders/load_gltf.cpp:12-315):

* meshes: TRIANGLES primitives with POSITION, optional NORMAL and TEXCOORD_0, indexed (the
  reference needs indices; non-indexed primitives get sequential ones); one instance per mesh
  primitive under every node that references the mesh, with the node's world transform (matrix or
  TRS, parents first);
* materials: makeMetallicRoughnessMaterial (src/App/Scene.cpp:195-208) from the
  pbrMetallicRoughness factors, emissiveFactor x KHR_materials_emissive_strength,
  KHR_materials_ior (default 1.5), KHR_materials_transmission, then KHR_materials_clearcoat and
  KHR_materials_specular (load_gltf.cpp:92-128); the normal texture is the bump image (strength 1);
* textures: PNG (the decoder below, 8-bit) and JPEG (Pillow's decoder: the reference decodes with
  stb_image through tinygltf, whose JPEG IDCT and chroma upsampling may differ from libjpeg's by one
  8-bit step), expanded to RGBA8; repacked per texel into the four packed-material images on the
  GPU (Device.repack_metallic_roughness, the reference's from_gltf_pbr pass,
  convert_material.slang:33-69), which decodes the base colour and emission as sRGB, with the base
  colour's alpha as the alpha mask;
* cameras: perspective cameras become views (make_view) at their node's position and rotation.
"""
from __future__ import annotations

import base64
import json
import math
import struct
import zlib
from pathlib import Path

import numpy as np

from . import _abi
from .scene import Material, Scene, make_view, rotation_from_quaternion

_COMPONENT = {5120: np.int8, 5121: np.uint8, 5122: np.int16, 5123: np.uint16, 5125: np.uint32, 5126: np.float32}
_NCOMP = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT4": 16}


# ------------------------------------------------------------------------------ PNG
PNG_MAGIC = b"\x89PNG\r\n\x1a\n"
JPEG_MAGIC = b"\xff\xd8\xff"


def decode_png_rgba8(data: bytes) -> np.ndarray:
    """8-bit PNG (grey, RGB, palette, grey + alpha, RGBA; no interlace) -> uint8 (h, w, 4), grey
    broadcast to RGB, alpha 255 where the image has none."""
    if data[:8] != PNG_MAGIC:
        raise ValueError("not a PNG image")
    pos, idat, plte, trns = 8, b"", None, None
    w = h = depth = ctype = interlace = None
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        pos += 12 + n
        if kind == b"IHDR":
            w, h, depth, ctype, _, _, interlace = struct.unpack(">IIBBBBB", body)
        elif kind == b"PLTE":
            plte = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif kind == b"tRNS":
            trns = np.frombuffer(body, np.uint8)
        elif kind == b"IDAT":
            idat += body
        elif kind == b"IEND":
            break
    if depth != 8 or interlace:
        raise ValueError("only 8-bit, non-interlaced PNG images are supported")
    ch = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + w * ch)
    out = np.zeros((h, w * ch), np.int32)
    prev = np.zeros(w * ch, np.int32)
    for y in range(h):
        f, line = raw[y, 0], raw[y, 1:].astype(np.int32)
        cur = np.zeros(w * ch, np.int32)
        if f == 0:
            cur = line
        elif f == 2:
            cur = (line + prev) & 0xFF
        else:
            for x in range(w * ch):
                a = cur[x - ch] if x >= ch else 0
                b = prev[x]
                c = prev[x - ch] if x >= ch else 0
                if f == 1:
                    pred = a
                elif f == 3:
                    pred = (a + b) >> 1
                else:  # Paeth
                    p = a + b - c
                    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                    pred = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
                cur[x] = (line[x] + pred) & 0xFF
        out[y] = cur
        prev = cur
    px = out.reshape(h, w, ch).astype(np.uint8)
    rgba = np.full((h, w, 4), 255, np.uint8)
    if ctype == 3:
        rgba[..., :3] = plte[px[..., 0]]
        if trns is not None:
            alpha = np.full(256, 255, np.uint8)
            alpha[:len(trns)] = trns
            rgba[..., 3] = alpha[px[..., 0]]
    elif ch == 1:
        rgba[..., :3] = px
    elif ch == 2:
        rgba[..., :3] = px[..., :1]
        rgba[..., 3] = px[..., 1]
    else:
        rgba[..., :ch] = px
    return rgba


def decode_png(data: bytes) -> np.ndarray:
    """decode_png_rgba8 as float32 in [0, 1]."""
    return decode_png_rgba8(data).astype(np.float32) / np.float32(255.0)


def decode_jpeg_rgba8(data: bytes) -> np.ndarray:
    """Baseline or progressive JPEG (grey, YCbCr, CMYK) -> uint8 (h, w, 4), alpha 255."""
    import io

    from PIL import Image
    with Image.open(io.BytesIO(data)) as im:
        if im.format != "JPEG":
            raise ValueError("not a JPEG image")
        return np.asarray(im.convert("RGBA"), np.uint8).copy()


def decode_image_rgba8(data: bytes) -> np.ndarray:
    """A glTF image (PNG or JPEG, by its signature) -> uint8 (h, w, 4)."""
    if data[:8] == PNG_MAGIC:
        return decode_png_rgba8(data)
    if data[:3] == JPEG_MAGIC:
        return decode_jpeg_rgba8(data)
    raise ValueError("unsupported image format (PNG and JPEG are supported)")


# ------------------------------------------------------------------------------ loader
class GltfScene:
    def __init__(self, scene: Scene, views: list, instances: int):
        self.scene, self.views, self.instances = scene, views, instances


def _trs_matrix(node) -> np.ndarray:
    if "matrix" in node:
        return np.asarray(node["matrix"], np.float64).reshape(4, 4).T  # column-major
    m = np.eye(4)
    t = node.get("translation", [0, 0, 0])
    r = node.get("rotation", [0, 0, 0, 1])  # x, y, z, w
    s = node.get("scale", [1, 1, 1])
    rot = rotation_from_quaternion(tuple(r))  # glTF order x, y, z, w
    m[:3, :3] = np.asarray(rot, np.float64) @ np.diag(s)
    m[:3, 3] = t
    return m


def load_gltf(path, width: int = 640, height: int = 480, device=None, repack=None) -> GltfScene:
    """Loads a .gltf or .glb file.  Textured materials are repacked on the GPU through `device`
    (a Device); `repack` replaces that call (same signature and result as
    Device.repack_metallic_roughness).  A textured material with neither raises ValueError."""
    path = Path(path)
    if repack is None and device is not None:
        repack = device.repack_metallic_roughness
    raw = path.read_bytes()
    bin_chunk = None
    if raw[:4] == b"glTF":
        _, version, total = struct.unpack("<III", raw[:12])
        pos, doc = 12, None
        while pos < total:
            n, kind = struct.unpack("<II", raw[pos:pos + 8])
            body = raw[pos + 8:pos + 8 + n]
            if kind == 0x4E4F534A:
                doc = json.loads(body.decode("utf-8"))
            elif kind == 0x004E4942:
                bin_chunk = body
            pos += 8 + n
    else:
        doc = json.loads(raw.decode("utf-8"))

    def buffer_bytes(i):
        b = doc["buffers"][i]
        uri = b.get("uri")
        if uri is None:
            return bin_chunk
        if uri.startswith("data:"):
            return base64.b64decode(uri.split(",", 1)[1])
        return (path.parent / uri).read_bytes()

    buffers = [buffer_bytes(i) for i in range(len(doc.get("buffers", [])))]

    def view_bytes(vi):
        v = doc["bufferViews"][vi]
        b = buffers[v["buffer"]]
        off = v.get("byteOffset", 0)
        return b[off:off + v["byteLength"]], v.get("byteStride")

    def accessor(ai):
        a = doc["accessors"][ai]
        dt = np.dtype(_COMPONENT[a["componentType"]])
        nc = _NCOMP[a["type"]]
        count = a["count"]
        data, stride = view_bytes(a["bufferView"])
        off = a.get("byteOffset", 0)
        stride = stride or dt.itemsize * nc
        rows = np.frombuffer(data, np.uint8, count=(count - 1) * stride + dt.itemsize * nc, offset=off)
        arr = np.lib.stride_tricks.as_strided(rows, (count, dt.itemsize * nc), (stride, 1)).copy()
        arr = arr.view(dt).reshape(count, nc)
        if a.get("normalized") and dt.kind in "iu":
            arr = arr.astype(np.float32) / np.iinfo(dt).max
        return arr

    image_cache = {}

    def texture(tex_info):
        """The texture's image as decoded RGBA8 (the sRGB decode is the repack's)."""
        if tex_info is None:
            return None
        t = doc["textures"][tex_info["index"]]
        key = t["source"]
        if key not in image_cache:
            im = doc["images"][t["source"]]
            if "bufferView" in im:
                data, _ = view_bytes(im["bufferView"])
            elif im["uri"].startswith("data:"):
                data = base64.b64decode(im["uri"].split(",", 1)[1])
            else:
                data = (path.parent / im["uri"]).read_bytes()
            image_cache[key] = decode_image_rgba8(bytes(data))
        return image_cache[key]

    s = Scene()
    mat_addr = []
    for gm in doc.get("materials", []):
        pbr = gm.get("pbrMetallicRoughness", {})
        ext = gm.get("extensions", {})
        bc = pbr.get("baseColorFactor", [1, 1, 1, 1])[:3]
        rough, metal = pbr.get("roughnessFactor", 1.0), pbr.get("metallicFactor", 1.0)
        em = np.asarray(gm.get("emissiveFactor", [0, 0, 0]), np.float64)
        if "KHR_materials_emissive_strength" in ext:
            em = em * ext["KHR_materials_emissive_strength"].get("emissiveStrength", 1.0)
        eta = ext.get("KHR_materials_ior", {}).get("ior", 1.5)
        trans = ext.get("KHR_materials_transmission", {}).get("transmissionFactor", 0.0)
        m = Material.metallic_roughness(bc, rough, metal, emission=tuple(em), transmission=trans, eta=eta)
        if "KHR_materials_clearcoat" in ext:
            m.clearcoat = ext["KHR_materials_clearcoat"].get("clearcoatFactor", 0.0)
        if "KHR_materials_specular" in ext:
            sp = ext["KHR_materials_specular"]
            if "specularColorFactor" in sp:
                c = sp["specularColorFactor"]
                m.specular = 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]
            elif "specularFactor" in sp:
                m.specular = sp["specularFactor"]
        base_t = texture(pbr.get("baseColorTexture"))
        mr_t = texture(pbr.get("metallicRoughnessTexture"))
        em_t = texture(gm.get("emissiveTexture"))
        present = [t for t in (base_t, mr_t, em_t) if t is not None]
        if present:
            if repack is None:
                raise ValueError("textured glTF materials are repacked on the GPU: pass device=")
            if len({t.shape for t in present}) != 1:
                raise ValueError("the textures of one material must share one extent")
            imgs, alpha, min_alpha = repack(base_t, mr_t, em_t)
            ids = [s.add_image(imgs[0]), s.add_image(imgs[1]) if em_t is not None else _abi.NO_IMAGE,
                   s.add_image(imgs[2]) if mr_t is not None else _abi.NO_IMAGE, _abi.NO_IMAGE]
            m.images = tuple(ids)
            if alpha is not None and min_alpha < 255:
                m.alpha_mask = s.add_image(alpha)
        nt = gm.get("normalTexture")
        if nt is not None:
            m.bump_image = s.add_image(texture(nt)[..., :3].astype(np.float32) / np.float32(255.0))
            m.bump_strength = 1.0
            m.bump_channels = 3
        mat_addr.append(s.add_material(m))
    default_mat = None

    meshes = []
    for gmesh in doc.get("meshes", []):
        prims = []
        for pr in gmesh["primitives"]:
            if pr.get("mode", 4) != 4:
                continue  # only triangle lists
            attr = pr["attributes"]
            pos = accessor(attr["POSITION"]).astype(np.float32)
            idx = accessor(pr["indices"]).reshape(-1, 3).astype(np.uint32) if "indices" in pr else \
                np.arange(len(pos), dtype=np.uint32).reshape(-1, 3)
            nrm = accessor(attr["NORMAL"]).astype(np.float32) if "NORMAL" in attr else None
            uv = accessor(attr["TEXCOORD_0"]).astype(np.float32) if "TEXCOORD_0" in attr else None
            prims.append((s.add_mesh(pos, idx, normals=nrm, uvs=uv), pr.get("material")))
        meshes.append(prims)

    views, count = [], 0
    roots = doc.get("scenes", [{"nodes": list(range(len(doc.get("nodes", []))))}])[doc.get("scene", 0)]["nodes"]
    stack = [(n, np.eye(4)) for n in reversed(roots)]
    while stack:
        ni, parent = stack.pop()
        node = doc["nodes"][ni]
        world = parent @ _trs_matrix(node)
        if "mesh" in node:
            for mesh, mat in meshes[node["mesh"]]:
                if mat is None:
                    if default_mat is None:
                        default_mat = s.add_material(Material.metallic_roughness((1, 1, 1), 1.0, 1.0))
                    addr = default_mat
                else:
                    addr = mat_addr[mat]
                s.add_instance(mesh, addr, world[:3, :4].astype(np.float32))
                count += 1
        if "camera" in node:
            cam = doc["cameras"][node["camera"]]
            if cam.get("type") == "perspective":
                rot = world[:3, :3] / np.linalg.norm(world[:3, :3], axis=0, keepdims=True)
                views.append(make_view(tuple(world[:3, 3]), width, height, math.degrees(cam["perspective"]["yfov"]), rot))
        for c in reversed(node.get("children", [])):
            stack.append((c, world))
    return GltfScene(s, views, count)
