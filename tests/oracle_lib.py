"""ctypes access to the oracle (oracle/liboracle.so) and to the reference compat probe
(oracle/_ref/libref_compat.so).  Test infrastructure only."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE = ROOT / "oracle" / "liboracle.so"
REF = ROOT / "oracle" / "_ref" / "libref_compat.so"

_o = None
_r = None


def oracle() -> C.CDLL:
    global _o
    if _o is None:
        if not ORACLE.exists():
            import sys
            sys.path.insert(0, str(ROOT / "oracle"))
            from build_oracle import build_oracle  # noqa: E402
            build_oracle()
        L = C.CDLL(str(ORACLE))
        P = C.POINTER
        L.oracle_scene_create.restype = C.c_void_p
        L.oracle_scene_create.argtypes = [C.c_void_p, C.c_int]
        L.oracle_scene_destroy.argtypes = [C.c_void_p]
        L.oracle_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.oracle_render.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_int]
        L.oracle_pcg4d.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        L.oracle_math.argtypes = [C.c_int, C.c_void_p, C.c_uint32, C.c_void_p, C.c_int]
        L.oracle_env_eval.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        L.oracle_pack_normal.restype = C.c_uint32
        L.oracle_pack_normal.argtypes = [C.c_double, C.c_double, C.c_double]
        L.oracle_unpack_normal.argtypes = [C.c_uint32, C.c_void_p]
        L.oracle_half_round.restype = C.c_float
        L.oracle_half_round.argtypes = [C.c_float]
        L.oracle_bsdf_eval.argtypes = [C.c_void_p, C.c_float, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_bsdf_sample.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        _o = L
    return _o


REF_SHADER = ROOT / "oracle" / "_ref" / "libref_shader.so"
_rs = None

# Function ids shared by oracle_math, ref_shader_math and s2_device_math; 8 input and 9 output
# doubles per entry.
MATH_FUNCTIONS = ["xxhash32", "pcg", "pcg4d", "next_float", "pack_normal", "unpack_normal", "gtr1", "gtr2",
                  "smith_gtr2", "smith_gtr1", "vndf", "schlick", "fresnel_dielectric", "concentric_disc",
                  "cos_hemisphere", "uniform_sphere", "uniform_triangle", "orthonormal"]
MATH_IN, MATH_OUT = 8, 9


def ref_shader() -> C.CDLL | None:
    """The reference's shader math compiled as host C++ (oracle/build_oracle.py build_ref_shader)."""
    global _rs
    if _rs is None:
        if not REF_SHADER.exists():
            return None
        L = C.CDLL(str(REF_SHADER))
        L.ref_shader_math.argtypes = [C.c_int, C.c_void_p, C.c_uint32, C.c_void_p]
        _rs = L
    return _rs


def math_inputs(fn: int, n: int, seed: int) -> np.ndarray:
    """Seeded inputs (n, 8) in each function's domain."""
    rng = np.random.default_rng(seed + 101 * fn)
    a = np.zeros((n, MATH_IN))
    name = MATH_FUNCTIONS[fn]
    unit = rng.normal(size=(n, 3))
    unit /= np.linalg.norm(unit, axis=1, keepdims=True)
    u32 = lambda k: rng.integers(0, 2 ** 32, size=(n, k), dtype=np.uint64).astype(np.float64)
    uni = lambda k: rng.uniform(0.0, 1.0, size=(n, k)).astype(np.float32).astype(np.float64)
    if name in ("xxhash32", "pcg"):
        a[:, :1] = u32(1)
    elif name in ("pcg4d", "next_float"):
        a[:, :4] = u32(4)
    elif name == "pack_normal":
        a[:, :3] = unit
    elif name == "unpack_normal":
        a[:, 0] = (rng.integers(0, 2 ** 16, n) | (rng.integers(0, 2 ** 16, n) << 16)).astype(np.float64)
    elif name == "gtr1":
        a[:, 0] = rng.uniform(0.0, 1.0, n)
        a[:, 1] = rng.uniform(0.001, 0.99, n)
    elif name in ("gtr2", "smith_gtr2"):
        a[:, :3] = np.where(unit[:, 2:3] < 0, unit * [1, 1, -1], unit) if name == "gtr2" else unit
        a[:, 3:5] = rng.uniform(0.01, 1.0, (n, 2))
    elif name == "smith_gtr1":
        a[:, :3] = unit
    elif name == "vndf":
        a[:, :3] = unit
        a[:, 3:5] = rng.uniform(0.01, 1.0, (n, 2))
        a[:, 5:7] = uni(2)
    elif name == "schlick":
        a[:, 0] = rng.uniform(0.0, 1.0, n)
        a[:, 1] = rng.uniform(-0.2, 1.0, n)
    elif name == "fresnel_dielectric":
        a[:, 0] = rng.uniform(-1.0, 1.0, n)
        a[:, 1] = rng.uniform(0.5, 2.5, n)
    elif name in ("concentric_disc", "cos_hemisphere", "uniform_sphere", "uniform_triangle"):
        a[:, :2] = uni(2)
    elif name == "orthonormal":
        a[:, :3] = unit
        a[: n // 8, :3] = np.array([1.0, 1.0, 1.0]) / np.sqrt(3.0)  # the branch for N with equal components
    return a


def ref_compat() -> C.CDLL | None:
    global _r
    if _r is None:
        if not REF.exists():
            return None
        L = C.CDLL(str(REF))
        L.ref_pack_material.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_unpack_material.argtypes = [C.c_void_p, C.c_float, C.c_void_p]
        L.ref_mesh_instance.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p]
        L.ref_vertex_info.argtypes = [C.c_void_p, C.c_void_p]
        L.ref_make_perspective.argtypes = [C.c_float, C.c_float, C.c_float, C.c_void_p]
        L.ref_back_project.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_void_p]
        L.ref_sizes.argtypes = [C.c_void_p]
        _r = L
    return _r


def default_render_params():
    """Render parameters with the reference's defaults (TestRenderer.cpp:38-43, 52: maxDepth 5,
    environment sample probability 0.9, 32 RIS candidates, M cap 3, 100,000 hash-grid cells of size
    0.5), filled on the host without loading the product library."""
    from stratum2_b200 import _abi
    p = _abi.S2RenderParams()
    p.min_path_length, p.max_path_length, p.exposure, p.spp = 0, 5, 0.0, 1
    p.environment_sample_probability = 0.9
    p.restir_candidates = 32
    p.restir_max_m = 3.0
    p.restir_grid_cells = 100000
    p.restir_grid_cell_size = 0.5
    return p


class OracleScene:
    """An oracle copy of a packed scene (precision_mask: 1 = FP64, 2 = FP32-exact, 3 = both)."""

    def __init__(self, scene, precision_mask: int = 3):
        self._desc = scene.desc()
        self.h = oracle().oracle_scene_create(C.byref(self._desc), precision_mask)
        assert self.h

    def __del__(self):
        try:
            oracle().oracle_scene_destroy(self.h)
        except Exception:
            pass

    def trace(self, rays: np.ndarray, anyhit: bool = False, precision: int = 64, threads: int = 0) -> dict:
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        t = np.zeros(n)
        inst = np.zeros(n, np.uint32)
        prim = np.zeros(n, np.uint32)
        b1 = np.zeros(n)
        b2 = np.zeros(n)
        rc = oracle().oracle_trace(self.h, rays.ctypes.data, n, int(anyhit), precision, t.ctypes.data,
                                   inst.ctypes.data, prim.ctypes.data, b1.ctypes.data, b2.ctypes.data, threads)
        assert rc == 0
        return {"t": t, "instance": inst, "primitive": prim, "b1": b1, "b2": b2}

    def env_eval(self, params, dirs: np.ndarray):
        """Environment radiance (n, 3) and light-sampling solid-angle pdf (n,) of unit directions
        (n, 3), FP64 scene."""
        dirs = np.ascontiguousarray(dirs, np.float64)
        n = dirs.shape[0]
        rgb, pdf = np.zeros((n, 3)), np.zeros(n)
        assert oracle().oracle_env_eval(self.h, C.byref(params), dirs.ctypes.data, n, rgb.ctypes.data, pdf.ctypes.data) == 0
        return rgb, pdf

    def render(self, view, params, width: int, height: int, precision: int = 64, rect=None, stride: int = 1,
               threads: int = 0) -> dict:
        x0, y0, x1, y1 = rect if rect is not None else (0, 0, width, height)
        n = width * height
        out = {
            "sum": np.zeros((height, width, 3)), "sumsq": np.zeros((height, width, 3)),
            "albedo": np.zeros((height, width, 4), np.float32), "visibility": np.zeros((height, width, 2), np.uint32),
            "depth": np.zeros((height, width, 4), np.float32), "prev_uv": np.zeros((height, width, 2), np.float32),
            "ids32": np.zeros((height, width, 2), np.uint32),
        }
        cnt = np.zeros(2, np.uint64)
        rc = oracle().oracle_render(self.h, C.byref(view), C.byref(params), precision, x0, y0, x1, y1, stride,
                                    out["sum"].ctypes.data, out["sumsq"].ctypes.data, out["albedo"].ctypes.data,
                                    out["visibility"].ctypes.data, out["depth"].ctypes.data,
                                    out["prev_uv"].ctypes.data, out["ids32"].ctypes.data, cnt.ctypes.data, threads)
        assert rc == 0
        out["extension_rays"] = int(cnt[0])
        out["shadow_rays"] = int(cnt[1])
        spp = max(params.spp, 1)
        out["mean"] = out["sum"] / spp
        out["var_of_mean"] = np.maximum(out["sumsq"] / spp - out["mean"] ** 2, 0) / max(spp - 1, 1)
        return out


def camera_rays(view, width: int, height: int) -> np.ndarray:
    """Pixel-centre camera rays of a view, generated on the host in float64 then rounded
    (used as seeded query rays, not as the renderer's own rays)."""
    proj = np.array(view.projection[:], np.float64)
    cam = np.array(view.camera_to_world[:], np.float64).reshape(3, 4)
    ys, xs = np.mgrid[0:height, 0:width]
    cx = 2 * (xs + 0.5) / width - 1
    cy = -(2 * (ys + 0.5) / height - 1)
    near = proj[4]
    sg = np.sign(near)
    d = np.stack([near * (cx * sg - proj[2]) / proj[0], near * (cy * sg - proj[3]) / proj[1],
                  np.full_like(cx, near)], -1).reshape(-1, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d = d @ cam[:, :3].T
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = np.broadcast_to(cam[:, 3], d.shape)
    r = np.zeros((d.shape[0], 8), np.float32)
    r[:, 0:3] = o
    r[:, 4:7] = d
    r[:, 7] = np.inf
    return r


def random_rays(n: int, seed: int, lo=-1.2, hi=1.2) -> np.ndarray:
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 4:7] = d
    r[:, 7] = np.inf
    return r
