"""Byte layouts of the packed scene, pinned against the reference's own compat headers
(src/Shaders/compat/*.h compiled by oracle/build_oracle.py into oracle/_ref/libref_compat.so)."""
import ctypes as C
import math
import struct

import numpy as np
import pytest

from oracle_lib import ref_compat
from stratum2_b200 import _abi
from stratum2_b200.scene import Material, Scene, make_view

pytestmark = pytest.mark.skipif(ref_compat() is None, reason="reference compat probe not built (reference tree absent)")


def test_struct_sizes():
    out = np.zeros(7, np.uint32)
    ref_compat().ref_sizes(out.ctypes.data)
    # InstanceData, MeshVertexInfo, TransformData, ProjectionData, ViewData, ShadingData, PackedMaterialData
    assert out[0] == 8 and out[1] == 32 and out[2] == 48 and out[3] == 32 and out[4] == 48 and out[5] == 48
    # the host struct is padded by Eigen's 16-byte uint4 alignment; the material buffer record
    # is written field by field by Material::store (src/App/Material.hpp:22-38)
    assert out[6] in (20, 32)
    assert C.sizeof(_abi.S2View) == 32 + 16 + 48 + 48  # ProjectionData + image rect + 2 transforms


@pytest.mark.parametrize("seed", range(4))
def test_material_packing_matches_reference(seed):
    rng = np.random.default_rng(seed)
    for _ in range(200):
        p = rng.uniform(-0.1, 1.1, 18).astype(np.float32)
        p[3:6] = rng.uniform(0, 20, 3) * (rng.uniform() < 0.5)
        words = np.zeros(4, np.uint32)
        scale = np.zeros(1, np.float32)
        ref_compat().ref_pack_material(p.ctypes.data, words.ctypes.data, scale.ctypes.data)
        m = Material(base_color=tuple(p[0:3]), emission=tuple(p[3:6]), specular=p[6], sheen=p[7], metallic=p[8],
                     roughness=p[9], anisotropic=p[10], subsurface=p[11], clearcoat=p[12], clearcoat_gloss=p[13],
                     transmission=p[14], eta=float(p[15]) + 1.0)
        mine, mscale = m.packed_words()
        if scale[0] > 0:
            assert list(words) == mine, (p, list(map(hex, words)), list(map(hex, mine)))
            assert np.float32(mscale) == scale[0]
        else:
            # zero emission: the reference divides 0/0 and casts NaN to an integer (undefined), so
            # only the words that do not hold emission are compared; the emission scale is 0
            assert scale[0] == 0 and mscale == 0
            assert int(words[0]) == mine[0] and int(words[2]) == mine[2] and int(words[3]) == mine[3]
            assert (int(words[1]) >> 24) == (mine[1] >> 24)
        rec = m.pack()
        assert len(rec) == 64
        assert struct.unpack("<4I", rec[:16]) == tuple(mine)


def test_material_getters_match_reference():
    rng = np.random.default_rng(7)
    L = ref_compat()
    for _ in range(100):
        words = rng.integers(0, 2 ** 32, 4, dtype=np.uint64).astype(np.uint32)
        out = np.zeros(16, np.float32)
        L.ref_unpack_material(words.ctypes.data, C.c_float(3.5), out.ctypes.data)
        w0 = int(words[0])
        assert out[0] == np.float32((w0 & 255) / np.float32(255))
        assert out[6] == np.float32(((w0 >> 24) & 255) / np.float32(255))
        assert abs(out[3] - ((int(words[1]) & 255) / 255.0) * 3.5) < 1e-6


def test_mesh_instance_and_vertex_info_match_reference():
    L = ref_compat()
    s = Scene()
    pos = np.random.default_rng(0).uniform(-1, 1, (30, 3))
    idx = np.arange(30).reshape(10, 3)
    uv = np.random.default_rng(1).uniform(0, 1, (30, 2))
    mesh = s.add_mesh(pos, idx, uvs=uv)
    addr = s.add_material(Material())
    s.add_instance(mesh, addr)
    out = np.zeros(2, np.uint32)
    L.ref_mesh_instance(addr, mesh.vertex_info_index, mesh.primitive_count, out.ctypes.data)
    assert tuple(out) == s.instances[0]
    vi = s.vertex_infos[0]
    args = np.array([vi[0] & 0xFFFF, 0, 2, vi[0] >> 16, 0, 12, vi[1] & 0xFFFF, 0, 0, vi[1] >> 16, 0, 8], np.uint32)
    ref = np.zeros(8, np.uint32)
    L.ref_vertex_info(args.ctypes.data, ref.ctypes.data)
    assert list(ref) == vi


def test_projection_and_back_projection_match_reference():
    L = ref_compat()
    out = np.zeros(8, np.float32)
    fovy = math.radians(40.0)
    L.ref_make_perspective(C.c_float(fovy), C.c_float(1.0), C.c_float(-0.001), out.ctypes.data)
    v = make_view((0, 0, 3), 256, 256, 40.0)
    mine = np.array(v.projection[:], np.float32)
    np.testing.assert_array_equal(out[[0, 1, 2, 3, 4, 7]], mine[[0, 1, 2, 3, 4, 7]])
    # ray through clip (0.3, -0.2) looks down -z
    bp = np.zeros(3, np.float32)
    L.ref_back_project(mine.ctypes.data, C.c_float(0.3), C.c_float(-0.2), bp.ctypes.data)
    assert bp[2] < 0 and bp[0] > 0 and bp[1] < 0
