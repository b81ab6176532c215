"""Seeded synthetic scenes with the sizes and value distributions of the benchmark configurations.

All scenes are generated from fixed seeds with numpy; nothing is read from disk.

  box_scene (1,000 random triangles in a closed box, ceiling quad light, Lambertian albedo
      U[0.2, 0.8], pinhole at (0,0,3), 40 degree FOV, 256x256, 16 spp, path length 2..5)
  terrain_scene (1024x1024 heightfield of 6-octave value noise, amplitude 0.2, plus 64 instanced
      level-5 icospheres (20,480 triangles each) under seeded transforms; GLTF metallic-roughness
      materials; 512x256 procedural HDR sky with a 5e3 sun lobe over a 0.5 degree cone;
      1920x1080, 64 spp, path length 3..12 with Russian roulette)
  cutout_scene (the box with normal-mapped, textured walls and an alpha-masked quad)
  terrain_scene(..., emissive_triangles=100_000) (the many-lights form: small one-sided emissive
      triangles hovering over the terrain, one instance each, power lognormal(0, 2))
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _abi
from .scene import Material, Scene, look_at_rotation, make_view, rotation_from_quaternion, transform_trs


@dataclass
class Workload:
    scene: Scene
    view: object
    width: int
    height: int
    spp: int
    min_path_length: int
    max_path_length: int
    lambertian: bool
    name: str


def quad(p0, p1, p2, p3):
    return np.array([p0, p1, p2, p3], np.float32), np.array([[0, 1, 2], [0, 2, 3]], np.uint32)


def box_scene(seed: int = 1, n_random: int = 1000, width: int = 256, height: int = 256, spp: int = 16,
              light_radiance: float = 10.0, closed: bool = True) -> Workload:
    """Closed box of 10 wall triangles spanning [-1,1]^3 (floor, ceiling, back, left, right),
    `n_random` random triangles inside, ceiling quad light 0.5x0.5 facing -y just below y=1."""
    rng = np.random.default_rng(seed)
    s = Scene()
    # walls: 5 faces x 2 triangles, normals pointing into the box
    walls = [
        ((-1, -1, -1), (-1, -1, 1), (1, -1, 1), (1, -1, -1)),   # floor (y=-1), normal +y
        ((-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)),       # ceiling (y=1), normal -y
        ((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)),   # back (z=-1), normal +z
        ((-1, -1, -1), (-1, 1, -1), (-1, 1, 1), (-1, -1, 1)),   # left (x=-1), normal +x
        ((1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)),       # right (x=1), normal -x
    ]
    wall_mat = s.add_material(Material(base_color=(0.7, 0.7, 0.7)))
    for w in walls:
        p, i = quad(*w)
        s.add_instance(s.add_mesh(p, i), wall_mat)
    # ceiling light facing -y
    h = 0.25
    y = 1.0 - 1e-3
    p, i = quad((-h, y, -h), (h, y, -h), (h, y, h), (-h, y, h))
    light_mat = s.add_material(Material(base_color=(0, 0, 0), emission=(light_radiance,) * 3))
    s.add_instance(s.add_mesh(p, i), light_mat)
    # random triangles, one instance (and material) per triangle for per-triangle albedo
    cent = rng.uniform(-0.8, 0.8, size=(n_random, 3))
    offs = rng.uniform(-0.05, 0.05, size=(n_random, 3, 3))
    alb = rng.uniform(0.2, 0.8, size=(n_random, 3))
    tri_idx = np.array([[0, 1, 2]], np.uint32)
    for k in range(n_random):
        verts = (cent[k][None, :] + offs[k]).astype(np.float32)
        m = s.add_material(Material(base_color=tuple(alb[k])))
        s.add_instance(s.add_mesh(verts, tri_idx), m)
    view = make_view((0.0, 0.0, 3.0), width, height, 40.0)
    return Workload(s, view, width, height, spp, 2, 5, True, f"box{n_random}_{width}x{height}")


def cutout_scene(seed: int = 3, n_random: int = 200, width: int = 64, height: int = 64, spp: int = 16) -> Workload:
    """The box with textured walls: floor and back wall carry a tangent-space normal map (3
    channels, strength 1) and an albedo texture; a 1.4 x 1.4 quad at z = 0.2 facing the camera has
    an alpha mask (R32F, 0 inside 12 random discs, 1 elsewhere, cutoff 0.5) so the random
    triangles behind it show through the holes."""
    rng = np.random.default_rng(seed)
    s = Scene()
    uv4 = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    # normal map from value-noise heights (RGB = 0.5 + 0.5 * (nx, -ny, nz): the reference flips y)
    hgt = value_noise(rng, 128, octaves=4, amplitude=1.0)
    gy, gx = np.gradient(hgt.astype(np.float64))
    n = np.stack([-gx * 8, -gy * 8, np.ones_like(gx)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    nmap = s.add_image(np.stack([0.5 + 0.5 * n[..., 0], 0.5 - 0.5 * n[..., 1], 0.5 + 0.5 * n[..., 2]], -1).astype(np.float32))
    tex = s.add_image(rng.uniform(0.3, 1.0, size=(32, 32, 3)).astype(np.float32))
    yy, xx = np.mgrid[0:64, 0:64] / 64.0
    mask = np.ones((64, 64), np.float32)
    for _ in range(12):
        cx, cy, r = rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), rng.uniform(0.05, 0.15)
        mask[(xx - cx) ** 2 + (yy - cy) ** 2 < r * r] = 0.0
    amask = s.add_image(mask)
    walls = [
        ((-1, -1, -1), (-1, -1, 1), (1, -1, 1), (1, -1, -1)),
        ((-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)),
        ((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)),
        ((-1, -1, -1), (-1, 1, -1), (-1, 1, 1), (-1, -1, 1)),
        ((1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)),
    ]
    bumpy = s.add_material(Material(base_color=(0.8, 0.8, 0.8), roughness=0.4, images=(tex, _abi.NO_IMAGE, _abi.NO_IMAGE, _abi.NO_IMAGE),
                                    bump_image=nmap, bump_strength=1.0, bump_channels=3))
    plain = s.add_material(Material(base_color=(0.7, 0.7, 0.7)))
    for k, w in enumerate(walls):
        p, i = quad(*w)
        s.add_instance(s.add_mesh(p, i, uvs=uv4 * 3.0), bumpy if k in (0, 2) else plain)
    h, y = 0.25, 1.0 - 1e-3
    p, i = quad((-h, y, -h), (h, y, -h), (h, y, h), (-h, y, h))
    s.add_instance(s.add_mesh(p, i), s.add_material(Material(base_color=(0, 0, 0), emission=(10.0,) * 3)))
    p, i = quad((-0.7, -0.7, 0.2), (0.7, -0.7, 0.2), (0.7, 0.7, 0.2), (-0.7, 0.7, 0.2))
    cut = s.add_material(Material(base_color=(0.9, 0.5, 0.2), roughness=0.3, alpha_mask=amask, alpha_cutoff=0.5))
    s.add_instance(s.add_mesh(p, i, uvs=uv4), cut)
    cent = rng.uniform(-0.8, 0.8, size=(n_random, 3))
    cent[:, 2] = rng.uniform(-0.9, 0.1, n_random)
    offs = rng.uniform(-0.08, 0.08, size=(n_random, 3, 3))
    alb = rng.uniform(0.2, 0.8, size=(n_random, 3))
    for k in range(n_random):
        m = s.add_material(Material(base_color=tuple(alb[k])))
        s.add_instance(s.add_mesh((cent[k][None, :] + offs[k]).astype(np.float32), np.array([[0, 1, 2]], np.uint32)), m)
    view = make_view((0.0, 0.0, 3.0), width, height, 40.0)
    return Workload(s, view, width, height, spp, 2, 5, False, f"cutout_{width}x{height}")


def textured_box_scene(seed: int = 4, n_random: int = 100, width: int = 48, height: int = 48, tex_res: int = 32,
                       env_res=(32, 16), spheres: int = 0, sphere_level: int = 3) -> Workload:
    """The box (open front) with textured walls for the differentiable renderer: floor, back and left
    walls take their base colour from an RGB albedo image (image 0) and their roughness from the y
    channel of a packed[2] image (image 1; material roughness 0 and metallic 0, so roughness =
    texel); a ceiling quad light; `n_random` small triangles and `spheres` icospheres (level
    `sphere_level`) inside; a small procedural sky (image 2) seen through the open front."""
    rng = np.random.default_rng(seed)
    s = Scene()
    albedo = s.add_image(rng.uniform(0.2, 0.9, (tex_res, tex_res, 3)).astype(np.float32))
    packed = np.ones((tex_res, tex_res, 4), np.float32)
    packed[..., 1] = rng.uniform(0.2, 0.9, (tex_res, tex_res))
    rough = s.add_image(packed)
    uv4 = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    walls = [
        ((-1, -1, -1), (-1, -1, 1), (1, -1, 1), (1, -1, -1)),
        ((-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)),
        ((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)),
        ((-1, -1, -1), (-1, 1, -1), (-1, 1, 1), (-1, -1, 1)),
        ((1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)),
    ]
    tex_mat = s.add_material(Material(base_color=(1, 1, 1), roughness=0.0, metallic=0.0, specular=0.5,
                                      images=(albedo, _abi.NO_IMAGE, rough, _abi.NO_IMAGE)))
    plain = s.add_material(Material(base_color=(0.7, 0.7, 0.7), roughness=0.6))
    for k, w in enumerate(walls):
        p, i = quad(*w)
        s.add_instance(s.add_mesh(p, i, uvs=uv4), tex_mat if k in (0, 2, 3) else plain)
    h, y = 0.25, 1.0 - 1e-3
    p, i = quad((-h, y, -h), (h, y, -h), (h, y, h), (-h, y, h))
    s.add_instance(s.add_mesh(p, i), s.add_material(Material(base_color=(0, 0, 0), emission=(10.0,) * 3)))
    cent = rng.uniform(-0.8, 0.8, size=(n_random, 3))
    offs = rng.uniform(-0.05, 0.05, size=(n_random, 3, 3))
    for k in range(n_random):
        m = s.add_material(Material(base_color=tuple(rng.uniform(0.2, 0.8, 3))))
        s.add_instance(s.add_mesh((cent[k][None, :] + offs[k]).astype(np.float32), np.array([[0, 1, 2]], np.uint32)), m)
    if spheres:
        sv, sf = icosphere(sphere_level)
        mesh = s.add_mesh(sv, sf)
        for k in range(spheres):
            c = rng.uniform(-0.75, 0.75, 3)
            r = rng.uniform(0.03, 0.12)
            m = s.add_material(Material(base_color=tuple(rng.uniform(0.2, 0.9, 3)), roughness=float(rng.uniform(0.2, 0.9))))
            s.add_instance(mesh, m, transform_trs(c, np.eye(3), (r, r, r)))
    s.set_environment((1.0, 1.0, 1.0), s.add_image(sky_image(env_res[0], env_res[1], sun_radiance=20.0, sun_cone_degrees=10.0)))
    view = make_view((0.0, 0.0, 3.0), width, height, 40.0)
    return Workload(s, view, width, height, 16, 0, 4, False, f"textured_box_{width}x{height}")


# ------------------------------------------------------------------------------ terrain
def value_noise(rng: np.random.Generator, n: int, octaves: int = 6, amplitude: float = 0.2) -> np.ndarray:
    """Sum of `octaves` octaves of bilinearly interpolated value noise on an n x n grid,
    lacunarity 2, gain 0.5, scaled so the total amplitude is `amplitude`."""
    h = np.zeros((n, n), np.float64)
    total = 0.0
    for o in range(octaves):
        cells = 4 * (2 ** o)
        lattice = rng.uniform(-1, 1, size=(cells + 1, cells + 1))
        x = np.linspace(0, cells, n, endpoint=False) + 0.5 * cells / n
        i0 = np.floor(x).astype(int)
        f = x - i0
        f = f * f * (3 - 2 * f)
        i1 = np.minimum(i0 + 1, cells)
        a = lattice[np.ix_(i0, i0)]
        b = lattice[np.ix_(i0, i1)]
        c = lattice[np.ix_(i1, i0)]
        d = lattice[np.ix_(i1, i1)]
        fx = f[None, :]
        fy = f[:, None]
        h += (0.5 ** o) * ((a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy)
        total += 0.5 ** o
    return (h / total * amplitude).astype(np.float32)


def icosphere(level: int):
    t = (1 + 5 ** 0.5) / 2
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = f
    for _ in range(level):
        cache = {}
        nf = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts, np.float32), np.array(faces, np.uint32)


def sky_image(width: int = 512, height: int = 256, sun_dir=(0.3, 0.8, 0.2), sun_radiance: float = 5e3,
              sun_cone_degrees: float = 0.5) -> np.ndarray:
    """Procedural HDR sky as an equirectangular image in the reference's spherical uv
    (compat/common.h:129-142): gradient from horizon to zenith plus a sun lobe of radiance
    `sun_radiance` over a cone of `sun_cone_degrees` (full angle)."""
    u = (np.arange(width) + 0.5) / width
    v = (np.arange(height) + 0.5) / height
    uu, vv = np.meshgrid(u, v)
    phi = (uu * 2 - 1) * math.pi
    theta = vv * math.pi
    d = np.stack([np.sin(theta) * np.cos(phi), np.cos(theta), np.sin(theta) * np.sin(phi)], -1)
    up = np.clip(d[..., 1], 0, 1)[..., None]
    horizon = np.array([0.9, 0.95, 1.0])
    zenith = np.array([0.25, 0.45, 0.9])
    ground = np.array([0.15, 0.13, 0.12])
    sky = np.where(d[..., 1:2] >= 0, horizon * (1 - up) + zenith * up, ground)
    s = np.asarray(sun_dir, np.float64)
    s /= np.linalg.norm(s)
    cosang = d @ s
    sun = (cosang >= math.cos(math.radians(sun_cone_degrees / 2))).astype(np.float64)[..., None] * sun_radiance
    img = np.concatenate([sky + sun * np.array([1.0, 0.95, 0.85]), np.ones((height, width, 1))], -1)
    return img.astype(np.float32)


def add_emissive_triangles(s: Scene, rng: np.random.Generator, hgt: np.ndarray, n: int, sigma: float, power: float,
                           height=(0.02, 0.08), edge_range=(0.01, 0.03)):
    """`n` small emissive triangles (edge in `edge_range`) hovering `height` above the heightfield
    `hgt` (spanning [-1,1] in x and z), each its own instance and material, emitting downwards
    (front face tilted up to 60 degrees from -y).  Emitted power (radiance x area x pi) is
    `power` x lognormal(0, sigma) with a random tint."""
    grid = hgt.shape[0]
    # canonical triangle in the xz plane; its front face (cross(v0 - v2, v1 - v2)) points to -y
    tri = np.array([[0.0, 0.0, 0.577], [0.5, 0.0, -0.289], [-0.5, 0.0, -0.289]], np.float32)
    nrm = np.cross(tri[0] - tri[2], tri[1] - tri[2])
    if nrm[1] > 0:
        tri = tri[[0, 2, 1]]
    mesh = s.add_mesh(tri, np.array([[0, 1, 2]], np.uint32))
    area1 = 0.5 * np.linalg.norm(np.cross(tri[0] - tri[2], tri[1] - tri[2]))
    xz = rng.uniform(-0.95, 0.95, size=(n, 2))
    gi = np.clip(np.round((xz + 1) / 2 * (grid - 1)).astype(int), 0, grid - 1)
    y = hgt[gi[:, 1], gi[:, 0]] + rng.uniform(height[0], height[1], n)
    edge = rng.uniform(edge_range[0], edge_range[1], n)
    tilt = np.arccos(rng.uniform(0.5, 1.0, n))
    azim = rng.uniform(0, 2 * np.pi, n)
    spin = rng.uniform(0, 2 * np.pi, n)
    pw = power * rng.lognormal(0.0, sigma, n)
    tint = rng.uniform(0.5, 1.0, size=(n, 3))
    for k in range(n):
        cs, sn = math.cos(spin[k]), math.sin(spin[k])
        r_spin = np.array([[cs, 0, sn], [0, 1, 0], [-sn, 0, cs]])
        ax = np.array([math.cos(azim[k]), 0.0, math.sin(azim[k])])   # tilt about a horizontal axis
        ct, st = math.cos(tilt[k]), math.sin(tilt[k])
        K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
        r_tilt = np.eye(3) + st * K + (1 - ct) * (K @ K)
        rot = r_tilt @ r_spin
        area = area1 * edge[k] ** 2
        radiance = pw[k] / (area * math.pi) * tint[k] / tint[k].max()
        m = s.add_material(Material(base_color=(0, 0, 0), emission=tuple(radiance)))
        s.add_instance(mesh, m, transform_trs((xz[k, 0], y[k], xz[k, 1]), rot, (edge[k],) * 3))


def terrain_scene(seed: int = 2, grid: int = 1024, spheres: int = 64, sphere_level: int = 5, width: int = 1920,
                  height: int = 1080, spp: int = 64, tiles: int = 16, area_lights: int = 0,
                  sun_radiance: float = 5e3, sun_cone_degrees: float = 0.5, emissive_triangles: int = 0,
                  emissive_sigma: float = 2.0, emissive_power: float = 2e-3, sky_scale: float = 1.0,
                  emissive_height=(0.02, 0.08), emissive_edge=(0.01, 0.03)) -> Workload:
    rng = np.random.default_rng(seed)
    s = Scene()
    hgt = value_noise(rng, grid)
    xs = np.linspace(-1, 1, grid, dtype=np.float32)
    # terrain split into tiles x tiles instances (each <= 65,535 triangles, one material each)
    step = (grid - 1) // tiles
    for ty in range(tiles):
        for tx in range(tiles):
            x0, x1 = tx * step, (grid - 1 if tx == tiles - 1 else (tx + 1) * step)
            y0, y1 = ty * step, (grid - 1 if ty == tiles - 1 else (ty + 1) * step)
            nx, ny = x1 - x0 + 1, y1 - y0 + 1
            gx, gz = np.meshgrid(xs[x0:x1 + 1], xs[y0:y1 + 1])
            pos = np.stack([gx, hgt[y0:y1 + 1, x0:x1 + 1], gz], -1).reshape(-1, 3)
            ii, jj = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1))
            a = (jj * nx + ii).reshape(-1)
            b = a + 1
            c = a + nx
            d = c + 1
            idx = np.concatenate([np.stack([a, c, b], -1), np.stack([b, c, d], -1)], 0).astype(np.uint32)
            m = s.add_material(Material.metallic_roughness(rng.uniform(0.05, 0.95, 3), rng.uniform(0.05, 1.0),
                                                           float(rng.uniform() < 0.3)))
            s.add_instance(s.add_mesh(pos, idx), m)
    sv, sf = icosphere(sphere_level)
    sphere_mesh = s.add_mesh(sv, sf)
    for k in range(spheres):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        r = rng.uniform(0.03, 0.12)
        c = (rng.uniform(-0.9, 0.9), rng.uniform(0.2, 0.5), rng.uniform(-0.9, 0.9))
        m = s.add_material(Material.metallic_roughness(rng.uniform(0.05, 0.95, 3), rng.uniform(0.05, 1.0),
                                                       float(rng.uniform() < 0.3)))
        s.add_instance(sphere_mesh, m, transform_trs(c, rotation_from_quaternion(q), (r, r, r)))
    for k in range(area_lights):
        c = np.array([rng.uniform(-0.8, 0.8), rng.uniform(0.6, 0.9), rng.uniform(-0.8, 0.8)])
        h = 0.05
        p, i = quad(c + (-h, 0, -h), c + (h, 0, -h), c + (h, 0, h), c + (-h, 0, h))
        lm = s.add_material(Material(base_color=(0, 0, 0), emission=tuple(rng.uniform(5, 20, 3))))
        s.add_instance(s.add_mesh(p, i), lm)
    if emissive_triangles:
        add_emissive_triangles(s, rng, hgt, emissive_triangles, emissive_sigma, emissive_power, emissive_height,
                               emissive_edge)
    s.set_environment((sky_scale,) * 3, s.add_image(sky_image(sun_radiance=sun_radiance, sun_cone_degrees=sun_cone_degrees)))
    pos = (0.0, 0.9, 1.9)
    view = make_view(pos, width, height, 45.0, look_at_rotation(pos, (0.0, 0.0, 0.0)))
    return Workload(s, view, width, height, spp, 3, 12, False, f"terrain{grid}_{width}x{height}")


# ------------------------------------------------------------------------------ animated camera
def catmull_rom_views(width: int, height: int, frames: int = 32, seed: int = 5, center=(0.0, 0.9, 1.9),
                      spread=(0.3, 0.1, 0.2), target=(0.0, 0.0, 0.0), control_points: int = 6, vfov_degrees: float = 45.0,
                      looping: bool = False):
    """Camera animation along a seeded closed Catmull-Rom spline: `control_points` positions drawn
    uniformly within `spread` of `center`, the camera looking at `target`; one view per frame, each
    carrying the previous frame's camera transform for reprojection.  The first view's previous
    transform is its own, or with `looping` the last view's (for playing the loop repeatedly)."""
    rng = np.random.default_rng(seed)
    ctrl = np.asarray(center, np.float64) + rng.uniform(-1, 1, (control_points, 3)) * np.asarray(spread, np.float64)

    def position(t):
        seg = int(np.floor(t)) % control_points
        u = t - np.floor(t)
        p0, p1, p2, p3 = (ctrl[(seg + k - 1) % control_points] for k in range(4))
        # uniform Catmull-Rom: tangents (p2 - p0) / 2 and (p3 - p1) / 2
        return 0.5 * ((2 * p1) + (-p0 + p2) * u + (2 * p0 - 5 * p1 + 4 * p2 - p3) * u * u + (-p0 + 3 * p1 - 3 * p2 + p3) * u ** 3)

    views, prev = [], None
    for f in range(frames):
        pos = position(control_points * f / frames)
        rot = look_at_rotation(pos, target)
        m = transform_trs(pos, rot)
        views.append(make_view(pos, width, height, vfov_degrees, rot, prev_camera_to_world=prev if prev is not None else m))
        prev = m
    if looping:
        views[0] = make_view(position(0.0), width, height, vfov_degrees, look_at_rotation(position(0.0), target),
                             prev_camera_to_world=prev)
    return views
