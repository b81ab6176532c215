"""Scene packing in the reference's byte layouts.

Builds the buffers that Stratum2's Scene::updateFrameData uploads (src/App/Scene.cpp:428-791):
InstanceData/MeshInstanceData (src/Shaders/compat/scene.h:30-58), TransformData (row-major 3x4,
compat/transform.h:7), MeshVertexInfo (compat/scene.h:89-132), raw vertex/index byte buffers,
64-byte material records (src/App/Material.hpp:22-38) whose first 20 bytes are
PackedMaterialData (compat/material_data.h:12-73), the 16-byte environment record
(src/App/Scene.hpp:41-45) and the light maps (Scene.cpp:441-491).
"""
from __future__ import annotations

import ctypes as C
import math
import struct
from dataclasses import dataclass, field

import numpy as np

from . import _abi

INSTANCE_TYPE_MESH = 0


def unorm8(x: float) -> int:
    """floor(saturate(x)*255 + 0.5) in single precision (material_data.h:51-73)."""
    x32 = np.float32(min(max(float(x), 0.0), 1.0))
    return int(np.floor(x32 * np.float32(255.0) + np.float32(0.5)))


@dataclass
class Material:
    """Disney/GLTF material parameters as PackedMaterialData stores them (8-bit UNORM each)."""
    base_color: tuple = (0.8, 0.8, 0.8)
    emission: tuple = (0.0, 0.0, 0.0)
    specular: float = 0.5
    sheen: float = 0.0
    metallic: float = 0.0
    roughness: float = 0.5
    anisotropic: float = 0.0
    subsurface: float = 0.0
    clearcoat: float = 0.0
    clearcoat_gloss: float = 0.0
    transmission: float = 0.0
    eta: float = 1.5                     # stored as eta - 1 (Scene.cpp:206)
    images: tuple = (_abi.NO_IMAGE,) * 4  # baseColor, emission, packed[2], packed[3] modulators
    bump_image: int = _abi.NO_IMAGE
    bump_strength: float = 1.0
    bump_channels: int = 0
    alpha_mask: int = _abi.NO_IMAGE
    alpha_cutoff: float = 0.5

    @staticmethod
    def metallic_roughness(base_color, roughness, metallic, emission=(0, 0, 0), transmission=0.0, eta=1.5):
        """makeMetallicRoughnessMaterial (src/App/Scene.cpp:195-208)."""
        return Material(base_color=tuple(base_color), emission=tuple(emission), specular=1.0, sheen=0.0,
                        metallic=metallic, roughness=roughness, anisotropic=0.0, subsurface=0.0, clearcoat=0.0,
                        clearcoat_gloss=0.0, transmission=transmission, eta=eta)

    def packed_words(self) -> tuple[list[int], float]:
        """PackedMaterialData.mPackedData and mEmissionScale."""
        bc = [unorm8(c) for c in self.base_color]
        em = [float(np.float32(e)) for e in self.emission]
        scale = float(np.float32(max(em)))
        if scale > 0:
            emq = [unorm8(np.float32(e) / np.float32(scale)) for e in em]
        else:
            emq = [0, 0, 0]   # setEmission with max 0 divides 0/0 -> NaN -> saturate -> 0
        w0 = bc[0] | bc[1] << 8 | bc[2] << 16 | unorm8(self.specular) << 24
        w1 = emq[0] | emq[1] << 8 | emq[2] << 16 | unorm8(self.sheen) << 24
        w2 = unorm8(self.metallic) | unorm8(self.roughness) << 8 | unorm8(self.anisotropic) << 16 | unorm8(self.subsurface) << 24
        w3 = unorm8(self.clearcoat) | unorm8(self.clearcoat_gloss) << 8 | unorm8(self.transmission) << 16 | unorm8(self.eta - 1.0) << 24
        return [w0, w1, w2, w3], scale

    def pack(self) -> bytes:
        """Material::store: 4 packed words, 4 image indices, emission scale, bump image/strength/
        channels, alpha mask/cutoff, 2 pad words = 64 bytes."""
        words, scale = self.packed_words()
        return _pack_record(words, self.images, scale, self)

    def has_emission(self) -> bool:
        words, scale = self.packed_words()
        return scale > 0 and (words[1] & 0xFFFFFF) != 0


def _pack_record(words, images, scale, m: Material) -> bytes:
    rec = struct.pack("<4I", *words)
    rec += struct.pack("<4I", *[int(i) & 0xFFFFFFFF for i in images])
    rec += struct.pack("<f", scale)
    rec += struct.pack("<IfI", int(m.bump_image) & 0xFFFFFFFF, float(m.bump_strength), int(m.bump_channels))
    rec += struct.pack("<If", int(m.alpha_mask) & 0xFFFFFFFF, float(m.alpha_cutoff))
    rec += struct.pack("<2I", 0, 0)
    assert len(rec) == 64
    return rec


def transform_trs(translation=(0, 0, 0), rotation=np.eye(3), scale=(1, 1, 1)) -> np.ndarray:
    """Row-major 3x4 object-to-world matrix (TransformData)."""
    m = np.zeros((3, 4), np.float32)
    m[:, :3] = np.asarray(rotation, np.float64) @ np.diag(np.asarray(scale, np.float64))
    m[:, 3] = translation
    return m


def rotation_from_quaternion(q) -> np.ndarray:
    x, y, z, w = q
    n = x * x + y * y + z * z + w * w
    s = 2.0 / n
    return np.array([
        [1 - s * (y * y + z * z), s * (x * y - z * w), s * (x * z + y * w)],
        [s * (x * y + z * w), 1 - s * (x * x + z * z), s * (y * z - x * w)],
        [s * (x * z - y * w), s * (y * z + x * w), 1 - s * (x * x + y * y)],
    ])


@dataclass
class Mesh:
    vertex_info_index: int
    primitive_count: int


class Scene:
    """Accumulates meshes, materials, instances, lights and an environment map, then exposes
    them as the packed S2SceneDesc the C ABI (and the oracle) consume."""

    def __init__(self):
        self.vertex_buffers: list[np.ndarray] = []    # uint8 arrays
        self.vertex_infos: list[list[int]] = []
        self.material_data = bytearray()
        self.materials: list[Material] = []
        self.material_addresses: list[int] = []
        self._material_at: dict[int, Material] = {}
        self.instances: list[tuple[int, int]] = []
        self.primitive_counts: list[int] = []
        self.transforms: list[np.ndarray] = []
        self.instance_material: list[int] = []
        self.light_instance_map: list[int] = []
        self.instance_light_map: list[int] = []
        self.images: list[np.ndarray] = []
        self.environment_address = _abi.NO_ENVIRONMENT
        self._aabb_min = np.full(3, np.inf)
        self._aabb_max = np.full(3, -np.inf)
        self._keep = []

    # ---- geometry
    def add_mesh(self, positions, indices, normals=None, uvs=None) -> Mesh:
        positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        indices = np.ascontiguousarray(indices).reshape(-1, 3)
        stride16 = positions.shape[0] <= 0xFFFF
        idx = indices.astype(np.uint16 if stride16 else np.uint32)
        ib = self._add_buffer(idx)
        pb = self._add_buffer(positions)
        nb = self._add_buffer(np.ascontiguousarray(normals, np.float32).reshape(-1, 3)) if normals is not None else _abi.NO_BUFFER
        tb = self._add_buffer(np.ascontiguousarray(uvs, np.float32).reshape(-1, 2)) if uvs is not None else _abi.NO_BUFFER
        istride = 2 if stride16 else 4
        w0 = ib | pb << 16
        w1 = nb | tb << 16
        w2 = istride | 12 << 8 | (12 if normals is not None else 0) << 16 | (8 if uvs is not None else 0) << 24
        self.vertex_infos.append([w0, w1, w2, 0, 0, 0, 0, 0])
        return Mesh(len(self.vertex_infos) - 1, int(indices.shape[0]))

    def _add_buffer(self, arr: np.ndarray) -> int:
        self.vertex_buffers.append(np.frombuffer(np.ascontiguousarray(arr).tobytes(), np.uint8).copy())
        return len(self.vertex_buffers) - 1

    def add_material(self, m: Material) -> int:
        addr = len(self.material_data)
        self.material_data += m.pack()
        self.materials.append(m)
        self.material_addresses.append(addr)
        self._material_at[addr] = m
        return addr

    def add_instance(self, mesh: Mesh, material_address: int, transform=None) -> int:
        if transform is None:
            transform = transform_trs()
        transform = np.asarray(transform, np.float32).reshape(3, 4)
        idx = len(self.instances)
        data = (mesh.vertex_info_index & 0xFFFF) | (min(mesh.primitive_count, 0xFFFF) << 16)
        self.instances.append((INSTANCE_TYPE_MESH | (material_address << 4), data))
        self.primitive_counts.append(mesh.primitive_count)
        self.transforms.append(transform)
        self.instance_material.append(material_address)
        m = self._material_at[material_address]
        if m.has_emission():
            self.instance_light_map.append(len(self.light_instance_map))
            self.light_instance_map.append(idx)
        else:
            self.instance_light_map.append(_abi.INVALID_INDEX16)
        # scene bounds for the scene sphere (TestRenderer.cpp:458-461)
        vi = self.vertex_infos[mesh.vertex_info_index]
        pos = np.frombuffer(self.vertex_buffers[vi[0] >> 16].tobytes(), np.float32).reshape(-1, 3)
        w = pos.astype(np.float64) @ transform[:, :3].T.astype(np.float64) + transform[:, 3]
        self._aabb_min = np.minimum(self._aabb_min, w.min(0))
        self._aabb_max = np.maximum(self._aabb_max, w.max(0))
        return idx

    def add_image(self, texels: np.ndarray) -> int:
        t = np.ascontiguousarray(texels, np.float32)
        if t.ndim == 2:
            t = t[:, :, None]
        self.images.append(t)
        return len(self.images) - 1

    def set_environment(self, emission_scale=(1, 1, 1), image: int = _abi.NO_IMAGE):
        """EnvironmentMap::store (src/App/Scene.hpp:41-45): float3 scale + image index."""
        self.environment_address = len(self.material_data)
        self.material_data += struct.pack("<3fI", *[float(x) for x in emission_scale], int(image) & 0xFFFFFFFF)

    @property
    def light_count(self) -> int:
        return len(self.light_instance_map)

    @property
    def triangle_count(self) -> int:
        return int(sum(self.primitive_counts))

    def scene_sphere(self) -> np.ndarray:
        c = (self._aabb_max + self._aabb_min) / 2
        r = float(np.linalg.norm(self._aabb_max - c))
        return np.array([*c, r], np.float32)

    # ---- packed view for the C ABI
    def desc(self) -> _abi.S2SceneDesc:
        keep = []

        def arr(a, ctype):
            a = np.ascontiguousarray(a)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(ctype))

        d = _abi.S2SceneDesc()
        n = len(self.instances)
        d.instance_count = n
        d.instances = arr(np.array(self.instances, np.uint32).reshape(-1), C.c_uint32) if n else None
        d.primitive_counts = arr(np.array(self.primitive_counts, np.uint32), C.c_uint32) if n else None
        d.transforms = arr(np.stack(self.transforms).astype(np.float32).reshape(-1), C.c_float) if n else None
        d.inverse_transforms = None
        d.motion_transforms = None
        d.vertex_info_count = len(self.vertex_infos)
        d.vertex_infos = arr(np.array(self.vertex_infos, np.uint32).reshape(-1), C.c_uint32) if self.vertex_infos else None
        nb = len(self.vertex_buffers)
        d.vertex_buffer_count = nb
        ptrs = (C.c_void_p * max(nb, 1))(*[b.ctypes.data for b in self.vertex_buffers])
        sizes = (C.c_uint64 * max(nb, 1))(*[b.nbytes for b in self.vertex_buffers])
        keep += [ptrs, sizes, self.vertex_buffers]
        d.vertex_buffers = C.cast(ptrs, C.POINTER(C.c_void_p))
        d.vertex_buffer_bytes = C.cast(sizes, C.POINTER(C.c_uint64))
        mat = np.frombuffer(bytes(self.material_data), np.uint8).copy()
        keep.append(mat)
        d.material_bytes = len(mat)
        d.material_data = mat.ctypes.data if len(mat) else None
        d.light_count = len(self.light_instance_map)
        d.light_instance_map = arr(np.array(self.light_instance_map, np.uint32), C.c_uint32) if self.light_instance_map else None
        d.instance_light_map = arr(np.array(self.instance_light_map, np.uint32), C.c_uint32) if n else None
        d.environment_material_address = self.environment_address
        imgs = (_abi.S2Image * max(len(self.images), 1))()
        for i, t in enumerate(self.images):
            imgs[i].width = t.shape[1]
            imgs[i].height = t.shape[0]
            imgs[i].channels = t.shape[2]
            imgs[i].texels = t.ctypes.data_as(C.POINTER(C.c_float))
        keep += [imgs, self.images]
        d.image_count = len(self.images)
        d.images = C.cast(imgs, C.POINTER(_abi.S2Image))
        sph = self.scene_sphere() if n else np.zeros(4, np.float32)
        for i in range(4):
            d.scene_sphere[i] = float(sph[i])
        d._keep = keep  # keep host arrays alive as long as the descriptor
        return d


# ------------------------------------------------------------------------------ views
def make_view(position, width: int, height: int, vfov_degrees: float, rotation=np.eye(3),
              prev_camera_to_world=None) -> _abi.S2View:
    """Pinhole view: ViewData with ProjectionData::makePerspective (compat/transform.h:181-190)
    at near plane -0.001 (reversed z, camera looking down -z, src/main.cpp:116) and the camera
    TransformData.  Horizontal scale uses height/width so pixels are square."""
    v = _abi.S2View()
    fovy = math.radians(vfov_degrees)
    sy = 1.0 / math.tan(fovy / 2)
    proj = [sy * height / width, sy, 0.0, 0.0, -0.001, -10000.0, 0.0, fovy]
    ext_x = 2.0 / proj[0]
    ext_y = 2.0 / proj[1]
    proj[6] = abs(ext_x * ext_y)  # sensor area (Scene.hpp:59-61)
    for i, x in enumerate(proj):
        v.projection[i] = float(np.float32(x))
    v.image_min[0], v.image_min[1] = 0, 0
    v.image_max[0], v.image_max[1] = width, height
    m = transform_trs(position, rotation)
    for i, x in enumerate(m.reshape(-1)):
        v.camera_to_world[i] = float(x)
    prev = m if prev_camera_to_world is None else np.asarray(prev_camera_to_world, np.float32).reshape(3, 4)
    inv = np.zeros((3, 4), np.float64)
    r = prev[:, :3].astype(np.float64)
    ri = np.linalg.inv(r)
    inv[:, :3] = ri
    inv[:, 3] = -ri @ prev[:, 3]
    for i, x in enumerate(inv.astype(np.float32).reshape(-1)):
        v.prev_world_to_camera[i] = float(x)
    return v


def look_at_rotation(position, target, up=(0, 1, 0)) -> np.ndarray:
    """Camera rotation whose -z axis points from position to target."""
    f = np.asarray(target, np.float64) - np.asarray(position, np.float64)
    f /= np.linalg.norm(f)
    z = -f
    x = np.cross(np.asarray(up, np.float64), z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    return np.stack([x, y, z], axis=1)
