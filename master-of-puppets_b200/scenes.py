"""Seeded synthetic scenes for the CPU software-rasterizer frame path.

Every workload the tests and the benchmark render is built here, once, from a
seed, so that the reference CPU backend, the plain-C oracle and the CUDA
backend all consume byte-identical vertex/index arrays, matrices, materials,
textures and lights.

Vertex layout is the reference's fixed ``MopVertex`` (include/mop/types.h:58):
position f32x3, normal f32x3, colour RGBA f32x4, uv f32x2 = 12 floats, 48 B.
Matrices are column-major ``d[col*4+row]`` (include/mop/types.h:39).

The scene descriptions follow the workloads the project is measured on:

* ``config1``  800x600, ssaa 1, UV sphere 64x32 at (0,0.5,0) + 20x20 ground
  plane, one directional light, untextured GGX materials.
* ``config2``  1920x1080, ssaa 2, 256 mesh instances (icospheres subdiv 4-6 and
  64x128 tori) with random TRS, 1 directional + 4 point + 2 spot lights,
  1024^2 value-noise base-colour textures, procedural-sky IBL, ACES.
* ``config3``  1920x1080, ssaa 1: clipping/depth stress (near-plane
  stragglers, out-of-frustum triangles, coplanar pairs with distinct IDs).
* ``small_*``  reduced-size variants for fast parity tests.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Tuple

import numpy as np

LIGHT_DIRECTIONAL, LIGHT_POINT, LIGHT_SPOT = 0, 1, 2
POST_GAMMA, POST_TONEMAP, POST_VIGNETTE, POST_FOG, POST_FXAA = 1, 2, 4, 8, 16
DEFAULT_POST = POST_GAMMA | POST_FXAA  # reference viewport.c:646


@dataclasses.dataclass
class Mesh:
    vertices: np.ndarray          # float32 [V, 12]
    indices: np.ndarray           # uint32 [I]
    object_id: int
    transform: np.ndarray         # float32 [16], column-major
    metallic: float = 0.0
    roughness: float = 0.5
    has_material: bool = True
    texture: int = -1
    opacity: float = 1.0
    blend_mode: int = 0           # MopBlendMode set explicitly (0: opaque unless opacity < 1)

    @property
    def triangle_count(self) -> int:
        return int(self.indices.size // 3)


TEX_RGBA8, TEX_BC1, TEX_BC3, TEX_BC5, TEX_BC7 = 0, 1, 2, 3, 4  # MopTexFormat


@dataclasses.dataclass
class CompressedTexture:
    """A block-compressed texture as mop_tex_create receives it (reference
    include/mop/core/texture_pipeline.h:35-56): BC1 (8 bytes per 4x4 block),
    BC3 or BC5 (16 bytes), blocks in row-major order."""
    width: int
    height: int
    format: int
    data: np.ndarray              # uint8 blocks

    @property
    def block_bytes(self) -> int:
        return 8 if self.format == TEX_BC1 else 16


def bc_texture(rng: np.random.Generator, fmt: int, width: int, height: int) -> CompressedTexture:
    """Seeded random blocks: both endpoint orders of every block kind occur
    (four-colour / three-colour BC1, eight-step / six-step BC4), and every
    fourth block has equal endpoints."""
    bw, bh = (width + 3) // 4, (height + 3) // 4
    bs = 8 if fmt == TEX_BC1 else 16
    data = rng.integers(0, 256, (bw * bh, bs), dtype=np.uint8)
    for h in ([0] if fmt == TEX_BC1 else [0, 8]):
        colour = fmt == TEX_BC1 or (fmt == TEX_BC3 and h == 8)
        if colour:
            data[::4, h + 2:h + 4] = data[::4, h:h + 2]  # c1 = c0 (16-bit endpoints)
        else:
            data[::4, h + 1] = data[::4, h]              # a1 = a0
    return CompressedTexture(width, height, fmt, data.reshape(-1))


@dataclasses.dataclass
class InstancedMesh:
    """mop_viewport_add_instanced_mesh (reference viewport.c:3774-3858): one
    mesh drawn once per transform, all with one object ID, the default
    material (metallic 0, roughness 0.5), no texture, opaque; the core draws
    it in pass_instanced, after the transparent pass (viewport.c:3238-3240),
    with mvp = P * (V * instance) (cpu_backend.c:638-657)."""
    vertices: np.ndarray          # float32 [V, 12]
    indices: np.ndarray           # uint32 [I]
    object_id: int
    transforms: np.ndarray        # float32 [N, 16], column-major

    @property
    def triangle_count(self) -> int:
        return int(self.indices.size // 3) * int(self.transforms.shape[0])


@dataclasses.dataclass
class Light:
    type: int
    position: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    direction: Tuple[float, float, float] = (0.0, -1.0, 0.0)
    color: Tuple[float, float, float, float] = (1.0, 1.0, 1.0, 1.0)
    intensity: float = 1.0
    range: float = 0.0
    spot_inner_cos: float = 0.95
    spot_outer_cos: float = 0.85
    active: bool = True
    cast_shadows: bool = False    # MopLight.cast_shadows (drives the shadow pass)


@dataclasses.dataclass
class Scene:
    name: str
    width: int
    height: int
    ssaa: int
    eye: Tuple[float, float, float]
    target: Tuple[float, float, float]
    up: Tuple[float, float, float] = (0.0, 1.0, 0.0)
    fov_deg: float = 45.0
    near: float = 0.1
    far: float = 100.0
    clear: Tuple[float, float, float, float] = (0.12, 0.13, 0.16, 1.0)
    ambient: float = 0.25
    exposure: float = 1.0
    post_effects: int = DEFAULT_POST
    meshes: List[Mesh] = dataclasses.field(default_factory=list)
    textures: List[np.ndarray] = dataclasses.field(default_factory=list)  # uint8 [h, w, 4]
    lights: List[Light] = dataclasses.field(default_factory=list)
    env: int = 0                  # 0 none, 1 procedural sky IBL
    sun_dir: Tuple[float, float, float] = (0.5, 0.7, 0.3)
    turbidity: float = 3.0
    ground_albedo: float = 0.3
    env_rotation: float = 0.0
    env_intensity: float = 1.0
    smooth: bool = True           # MOP_SHADING_SMOOTH (viewport default)
    # MopFogParams ((r, g, b, a), near, far) for the MOP_POST_FOG bit; None: not set
    fog: Optional[Tuple[Tuple[float, float, float, float], float, float]] = None
    instanced: List[InstancedMesh] = dataclasses.field(default_factory=list)
    # mop_viewport_set_environment_background: the environment drawn behind the scene
    env_background: bool = False
    # mop_viewport_set_render_mode(MOP_RENDER_WIREFRAME): meshes other than ID 0 as lines
    wireframe: bool = False
    # the reference core's own viewports only: keep its hidden grid mesh, which wireframe
    # mode draws (as lines, depth test off) although its opacity is 0
    wireframe_grid: bool = False

    @property
    def samples(self) -> int:
        return self.width * self.ssaa * self.height * self.ssaa

    @property
    def pixels(self) -> int:
        return self.width * self.height

    @property
    def triangle_count(self) -> int:
        return (sum(m.triangle_count for m in self.meshes)
                + sum(im.triangle_count for im in self.instanced))


# --------------------------------------------------------------------------
# matrices (column-major float32)
# --------------------------------------------------------------------------

def mat_identity() -> np.ndarray:
    m = np.zeros(16, np.float32)
    m[0] = m[5] = m[10] = m[15] = 1.0
    return m


def mat_trs(translation, rot3x3, scale) -> np.ndarray:
    """World = T * R * S, computed in float64 then rounded once to float32.

    The result is just input data: both renderers receive the same float32
    matrix, so how it was produced does not affect parity.
    """
    m = np.zeros((4, 4), np.float64)
    m[:3, :3] = np.asarray(rot3x3, np.float64) * np.asarray(scale, np.float64)[None, :]
    m[:3, 3] = translation
    m[3, 3] = 1.0
    return m.T.reshape(16).astype(np.float32)  # column-major flatten


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


# --------------------------------------------------------------------------
# geometry
# --------------------------------------------------------------------------

def _pack(pos, nrm, col, uv) -> np.ndarray:
    v = np.zeros((pos.shape[0], 12), np.float32)
    v[:, 0:3] = pos
    v[:, 3:6] = nrm
    v[:, 6:10] = col
    v[:, 10:12] = uv
    return v


def uv_sphere(segments: int, rings: int, radius: float, color) -> Tuple[np.ndarray, np.ndarray]:
    """UV sphere with (rings+1)*(segments+1) vertices; the degenerate pole
    triangles are dropped, giving segments*(2*rings-2) triangles (3,968 for
    64x32)."""
    th = np.linspace(0.0, math.pi, rings + 1)
    ph = np.linspace(0.0, 2.0 * math.pi, segments + 1)
    T, P = np.meshgrid(th, ph, indexing="ij")
    n = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1).reshape(-1, 3)
    uv = np.stack([P / (2 * math.pi), T / math.pi], -1).reshape(-1, 2)
    col = np.tile(np.asarray(color, np.float32), (n.shape[0], 1))
    verts = _pack(n * radius, n, col, uv)
    idx = []
    for r in range(rings):
        for s in range(segments):
            a = r * (segments + 1) + s
            b = a + segments + 1
            if r != 0:
                idx += [a, a + 1, b]
            if r != rings - 1:
                idx += [a + 1, b + 1, b]
    return verts, np.asarray(idx, np.uint32)


def ground_plane(size: float, color) -> Tuple[np.ndarray, np.ndarray]:
    h = size * 0.5
    pos = np.array([[-h, 0, -h], [h, 0, -h], [h, 0, h], [-h, 0, h]], np.float32)
    nrm = np.tile(np.array([0, 1, 0], np.float32), (4, 1))
    col = np.tile(np.asarray(color, np.float32), (4, 1))
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    return _pack(pos, nrm, col, uv), np.array([0, 2, 1, 0, 3, 2], np.uint32)


def icosphere(subdiv: int, radius: float, color) -> Tuple[np.ndarray, np.ndarray]:
    """Icosahedron subdivided ``subdiv`` times: 20*4^subdiv triangles."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}
        nf = []

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    n = np.asarray(verts, np.float64)
    uv = np.stack([np.arctan2(n[:, 2], n[:, 0]) / (2 * math.pi) + 0.5,
                   np.arcsin(np.clip(n[:, 1], -1, 1)) / math.pi + 0.5], -1)
    col = np.tile(np.asarray(color, np.float32), (n.shape[0], 1))
    # Counter-clockwise seen from outside: the reference's front faces.
    idx = np.asarray(faces, np.uint32).reshape(-1)
    return _pack(n * radius, n, col, uv), idx


def torus(major_seg: int, minor_seg: int, R: float, r: float, color) -> Tuple[np.ndarray, np.ndarray]:
    """Torus with major_seg x minor_seg quads = 2*major*minor triangles."""
    u = np.linspace(0, 2 * math.pi, major_seg + 1)
    v = np.linspace(0, 2 * math.pi, minor_seg + 1)
    U, V = np.meshgrid(u, v, indexing="ij")
    cx, cz = np.cos(U), np.sin(U)
    pos = np.stack([(R + r * np.cos(V)) * cx, r * np.sin(V), (R + r * np.cos(V)) * cz], -1).reshape(-1, 3)
    nrm = np.stack([np.cos(V) * cx, np.sin(V), np.cos(V) * cz], -1).reshape(-1, 3)
    uv = np.stack([U / (2 * math.pi), V / (2 * math.pi)], -1).reshape(-1, 2)
    col = np.tile(np.asarray(color, np.float32), (pos.shape[0], 1))
    idx = []
    for i in range(major_seg):
        for j in range(minor_seg):
            a = i * (minor_seg + 1) + j
            b = a + minor_seg + 1
            idx += [a, a + 1, b, a + 1, b + 1, b]
    return _pack(pos, nrm, col, uv), np.asarray(idx, np.uint32)


def value_noise_texture(rng: np.random.Generator, size: int, cells: int = 16) -> np.ndarray:
    """Seeded value noise, RGBA8 [size, size, 4]."""
    grid = rng.random((cells + 1, cells + 1, 3))
    x = np.linspace(0, cells, size, endpoint=False)
    xi = x.astype(np.int64)
    xf = x - xi
    xf = xf * xf * (3 - 2 * xf)
    a = grid[xi][:, xi]
    b = grid[xi][:, xi + 1]
    c = grid[xi + 1][:, xi]
    d = grid[xi + 1][:, xi + 1]
    fx = xf[None, :, None]
    fy = xf[:, None, None]
    top = a * (1 - fx) + b * fx
    bot = c * (1 - fx) + d * fx
    rgb = top * (1 - fy) + bot * fy
    tex = np.empty((size, size, 4), np.uint8)
    tex[..., :3] = np.clip(rgb * 255.0 + 0.5, 0, 255).astype(np.uint8)
    tex[..., 3] = 255
    return tex


def _mat_rand(rng):
    return (float(rng.uniform(0.0, 1.0)), float(rng.uniform(0.05, 1.0)))


def _color(rng):
    return (*[float(c) for c in rng.uniform(0.0, 1.0, 3)], 1.0)


# --------------------------------------------------------------------------
# configurations
# --------------------------------------------------------------------------

def config1(seed: int = 1, width: int = 800, height: int = 600, ssaa: int = 1) -> Scene:
    rng = np.random.default_rng(seed)
    sc = Scene("config1", width, height, ssaa, eye=(0.0, 3.0, 8.0), target=(0.0, 0.0, 0.0),
               fov_deg=45.0, near=0.1, far=100.0)
    sc.lights.append(Light(LIGHT_DIRECTIONAL, direction=(-0.4, -0.9, -0.3), intensity=3.0))
    c = _color(rng)
    metallic, rough = _mat_rand(rng)
    v, i = uv_sphere(64, 32, 1.0, c)
    t = mat_identity()
    t[13] = 0.5
    sc.meshes.append(Mesh(v, i, 1, t, metallic, rough))
    c = _color(rng)
    metallic, rough = _mat_rand(rng)
    v, i = ground_plane(20.0, c)
    sc.meshes.append(Mesh(v, i, 2, mat_identity(), metallic, rough))
    return sc


def config2(seed: int = 2, width: int = 1920, height: int = 1080, ssaa: int = 2,
            instances: int = 256, tex_size: int = 1024, n_textures: int = 4) -> Scene:
    """Large static scene.  256 instances: one subdiv-6 and one subdiv-5
    icosphere, 6 tori 64x128 and 248 subdiv-4 icospheres (1,470,464 tris)."""
    rng = np.random.default_rng(seed)
    sc = Scene("config2", width, height, ssaa, eye=(28.0, 18.0, 36.0), target=(0.0, 0.0, 0.0),
               fov_deg=50.0, near=0.5, far=200.0, env=1, sun_dir=(0.4, 0.8, 0.35),
               turbidity=3.0, ground_albedo=0.3)
    sc.lights.append(Light(LIGHT_DIRECTIONAL, direction=(-0.3, -0.8, -0.5), intensity=2.5,
                           color=(1.0, 0.96, 0.9, 1.0)))
    for _ in range(4):
        p = tuple(float(x) for x in rng.uniform(-18, 18, 3))
        sc.lights.append(Light(LIGHT_POINT, position=p, intensity=float(rng.uniform(20, 80)),
                               color=(*[float(x) for x in rng.uniform(0.5, 1.0, 3)], 1.0)))
    for _ in range(2):
        p = rng.uniform(-15, 15, 3)
        p[1] = abs(p[1]) + 10.0
        d = -p / np.linalg.norm(p)
        sc.lights.append(Light(LIGHT_SPOT, position=tuple(float(x) for x in p),
                               direction=tuple(float(x) for x in d),
                               intensity=float(rng.uniform(100, 300)), range=0.0,
                               spot_inner_cos=0.95, spot_outer_cos=0.85,
                               color=(*[float(x) for x in rng.uniform(0.5, 1.0, 3)], 1.0)))
    for _ in range(n_textures):
        sc.textures.append(value_noise_texture(rng, tex_size))
    kinds = ["s6", "s5"] + ["torus"] * 6 + ["s4"] * (instances - 8)
    kinds = kinds[:instances]
    rng.shuffle(kinds)
    proto = {}
    for k in set(kinds):
        if k == "torus":
            proto[k] = torus(64, 128, 1.0, 0.35, (1, 1, 1, 1))
        else:
            proto[k] = icosphere(int(k[1]), 1.0, (1, 1, 1, 1))
    for n, k in enumerate(kinds):
        v, i = proto[k]
        v = v.copy()
        v[:, 6:10] = _color(rng)
        metallic, rough = _mat_rand(rng)
        t = rng.uniform(-20, 20, 3)
        s = float(math.exp(rng.uniform(math.log(0.2), math.log(3.0))))
        m = mat_trs(t, random_rotation(rng), (s, s, s))
        sc.meshes.append(Mesh(v, i, n + 1, m, metallic, rough, texture=int(rng.integers(0, n_textures))))
    return sc


def served_scene(seed: int, target_tris: int, tex_size: int = 1024, n_textures: int = 4,
                 width: int = 1280, height: int = 720) -> Scene:
    """A config-2-style scene of about target_tris triangles: the config-2
    lights, textures and materials over instances drawn 80% subdiv-4
    icospheres, 10% tori 64x128, 8% subdiv-5 and 2% subdiv-6 icospheres,
    added until the triangle count reaches the target."""
    rng = np.random.default_rng(seed)
    base = config2(seed=seed, width=width, height=height, ssaa=1, instances=0,
                   tex_size=tex_size, n_textures=n_textures)
    proto = {}
    tris = 0
    n = 0
    while tris < target_tris:
        u = rng.random()
        k = "s4" if u < 0.8 else ("torus" if u < 0.9 else ("s5" if u < 0.98 else "s6"))
        if k not in proto:
            proto[k] = torus(64, 128, 1.0, 0.35, (1, 1, 1, 1)) if k == "torus" else \
                icosphere(int(k[1]), 1.0, (1, 1, 1, 1))
        v, i = proto[k]
        v = v.copy()
        v[:, 6:10] = _color(rng)
        metallic, rough = _mat_rand(rng)
        t = rng.uniform(-20, 20, 3)
        sc = float(math.exp(rng.uniform(math.log(0.2), math.log(3.0))))
        m = mat_trs(t, random_rotation(rng), (sc, sc, sc))
        base.meshes.append(Mesh(v, i, n + 1, m, metallic, rough,
                                texture=int(rng.integers(0, n_textures))))
        tris += i.size // 3
        n += 1
    base.name = f"served{seed}"
    return base


def served_triangle_counts(n: int = 32, seed: int = 5, lo: int = 50_000, hi: int = 2_000_000):
    """Log-normal scene sizes clipped to [lo, hi] (median ~300k)."""
    rng = np.random.default_rng(seed)
    return [int(min(max(math.exp(rng.normal(math.log(300_000), 0.9)), lo), hi))
            for _ in range(n)]


def small_scene(seed: int = 7, width: int = 160, height: int = 120, ssaa: int = 1,
                n_meshes: int = 6, lights: str = "mixed", textured: bool = True,
                env: int = 0) -> Scene:
    """A few spheres/tori with mixed lights; seconds on the oracle."""
    rng = np.random.default_rng(seed)
    sc = Scene(f"small{seed}", width, height, ssaa, eye=(4.0, 3.0, 7.0), target=(0.0, 0.3, 0.0),
               fov_deg=50.0, near=0.1, far=50.0, env=env, sun_dir=(0.3, 0.8, 0.4))
    if lights != "none":
        sc.lights.append(Light(LIGHT_DIRECTIONAL, direction=(-0.4, -0.9, -0.3), intensity=2.0))
    if lights == "mixed":
        sc.lights.append(Light(LIGHT_POINT, position=(2.0, 2.0, 2.0), intensity=6.0,
                               color=(1.0, 0.8, 0.6, 1.0)))
        sc.lights.append(Light(LIGHT_POINT, position=(-2.0, 1.0, 1.0), intensity=4.0, range=6.0,
                               color=(0.6, 0.8, 1.0, 1.0)))
        sc.lights.append(Light(LIGHT_SPOT, position=(0.0, 4.0, 2.0), direction=(0.0, -1.0, -0.4),
                               intensity=20.0, spot_inner_cos=0.95, spot_outer_cos=0.8))
        sc.lights.append(Light(LIGHT_SPOT, position=(3.0, 3.0, -1.0), direction=(-0.6, -0.7, 0.2),
                               intensity=10.0, range=8.0, spot_inner_cos=0.9, spot_outer_cos=0.7,
                               active=True))
        sc.lights.append(Light(LIGHT_POINT, position=(0.0, 1.0, 0.0), intensity=50.0, active=False))
    if textured:
        sc.textures.append(value_noise_texture(rng, 64, 8))
    v, i = ground_plane(12.0, _color(rng))
    m, r = _mat_rand(rng)
    sc.meshes.append(Mesh(v, i, 1, mat_identity(), m, r))
    for n in range(n_meshes):
        c = _color(rng)
        if n % 3 == 2:
            v, i = torus(24, 12, 0.7, 0.25, c)
        elif n % 3 == 1:
            v, i = icosphere(2, 0.6, c)
        else:
            v, i = uv_sphere(16, 8, 0.6, c)
        t = rng.uniform(-2.5, 2.5, 3)
        t[1] = abs(t[1]) * 0.5 + 0.6
        s = float(rng.uniform(0.6, 1.4))
        mtx = mat_trs(t, random_rotation(rng), (s, s, s))
        m, r = _mat_rand(rng)
        tex = 0 if (textured and n % 2 == 0) else -1
        sc.meshes.append(Mesh(v, i, n + 2, mtx, m, r, texture=tex))
    return sc


def _quad(x0, y0, x1, y1, z, color, tilt=0.0):
    pos = np.array([[x0, y0, z + tilt * x0], [x1, y0, z + tilt * x1], [x1, y1, z + tilt * x1],
                    [x0, y1, z + tilt * x0]], np.float32)
    n = np.array([-tilt, 0.0, 1.0])
    n = n / np.linalg.norm(n)
    nrm = np.tile(n.astype(np.float32), (4, 1))
    col = np.tile(np.asarray(color, np.float32), (4, 1))
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    return _pack(pos, nrm, col, uv), np.array([0, 1, 2, 0, 2, 3], np.uint32)


def coplanar_scene(seed: int = 3, width: int = 192, height: int = 144) -> Scene:
    """Overlapping quads on shared planes with distinct object IDs: exact
    depth ties must resolve to the earliest draw (strict `<` test,
    reference rasterizer.c:1960), rounding differences to the nearer."""
    rng = np.random.default_rng(seed)
    sc = Scene("coplanar", width, height, 1, eye=(0.0, 0.0, 5.0), target=(0.0, 0.0, 0.0),
               fov_deg=50.0, near=0.1, far=50.0)
    sc.lights.append(Light(LIGHT_DIRECTIONAL, direction=(-0.2, -0.3, -1.0), intensity=2.0))
    oid = 1
    for plane_z, tilt in ((0.0, 0.0), (-0.5, 0.35)):
        for _ in range(5):
            x0, y0 = rng.uniform(-2.2, 0.2, 2)
            x1, y1 = x0 + rng.uniform(1.0, 2.5), y0 + rng.uniform(1.0, 2.5)
            v, i = _quad(float(x0), float(y0), float(x1), float(y1), plane_z, _color(rng), tilt)
            m, r = _mat_rand(rng)
            sc.meshes.append(Mesh(v, i, oid, mat_identity(), m, r))
            oid += 1
    return sc


def skin_vertices(verts: np.ndarray, joints: np.ndarray, weights: np.ndarray,
                  mats: np.ndarray) -> np.ndarray:
    """Linear blend skinning on the host, as the core does before
    buffer_update (mop_skin_apply, reference viewport.c:1572-1680): position
    = sum over the 4 influences of w * (M_j * p); normal = sum of w * (M_j's
    3x3 * n), then normalised.  verts [V, 12] float32, joints [V, 4] int,
    weights [V, 4] float32 (sum 1), mats [J, 16] column-major float32."""
    out = verts.copy()
    p = verts[:, 0:3].astype(np.float32)
    n = verts[:, 3:6].astype(np.float32)
    pos = np.zeros_like(p)
    nrm = np.zeros_like(n)
    for b in range(4):
        m = mats[joints[:, b]].reshape(-1, 4, 4).transpose(0, 2, 1)  # row-major per vertex
        w = weights[:, b:b + 1].astype(np.float32)
        tp = np.einsum("vij,vj->vi", m[:, :3, :3], p) + m[:, :3, 3]
        tn = np.einsum("vij,vj->vi", m[:, :3, :3], n)
        pos += w * tp.astype(np.float32)
        nrm += w * tn.astype(np.float32)
    ln = np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm = np.where(ln > 1e-8, nrm / np.maximum(ln, 1e-30), nrm)
    out[:, 0:3] = pos
    out[:, 3:6] = nrm
    return out


def config3(seed: int = 3, width: int = 1920, height: int = 1080, n_tris: int = 2_000_000,
            tris_per_mesh: int = 2000) -> Scene:
    """Clipping and depth stress: n_tris triangles with screen-space edge
    length log-uniform 0.1-8 px; 10 % straddle the near plane, 5 % lie
    outside the frustum, 20 % come in coplanar pairs (the same triangle in two
    meshes with different object IDs, so draw order decides the tie); 5 % are
    joint-skinned tubes (4 influences, 64 joints, weights normalised to 1,
    skinned on the host).  Camera at (0, 0, 10) looking at the origin."""
    rng = np.random.default_rng(seed)
    fov, near, far = 50.0, 0.5, 100.0
    sc = Scene("config3", width, height, 1, eye=(0.0, 0.0, 10.0), target=(0.0, 0.0, 0.0),
               fov_deg=fov, near=near, far=far)
    sc.lights.append(Light(LIGHT_DIRECTIONAL, direction=(-0.3, -0.6, -1.0), intensity=2.5))
    sc.lights.append(Light(LIGHT_POINT, position=(2.0, 3.0, 6.0), intensity=40.0))
    t = math.tan(math.radians(fov) * 0.5)
    aspect = width / height
    eye = np.array([0.0, 0.0, 10.0])

    def place(ndc_x, ndc_y, depth):
        return eye + depth[:, None] * np.stack([ndc_x * t * aspect, ndc_y * t,
                                                -np.ones_like(depth)], 1)

    def tris(n, kind):
        if kind == "straddle":
            d = np.full(n, near)
            x, y = rng.uniform(-0.95, 0.95, n), rng.uniform(-0.95, 0.95, n)
        elif kind == "outside":
            d = np.exp(rng.uniform(math.log(2.0), math.log(60.0), n))
            x = rng.choice([-1, 1], n) * rng.uniform(1.3, 3.0, n)
            y = rng.uniform(-2.0, 2.0, n)
        else:
            d = np.exp(rng.uniform(math.log(1.0), math.log(80.0), n))
            x, y = rng.uniform(-1.05, 1.05, n), rng.uniform(-1.05, 1.05, n)
        c = place(x, y, d)
        px = np.exp(rng.uniform(math.log(0.1), math.log(8.0), n))
        size = px * 2.0 * d * t / height
        a = rng.normal(size=(n, 3))
        a /= np.linalg.norm(a, axis=1, keepdims=True)
        b = rng.normal(size=(n, 3))
        b -= (b * a).sum(1, keepdims=True) * a
        b /= np.linalg.norm(b, axis=1, keepdims=True)
        ang = rng.uniform(0, 2 * math.pi, (n, 3)) + np.array([0, 2.1, 4.2])
        v = c[:, None, :] + size[:, None, None] * (np.cos(ang)[..., None] * a[:, None, :]
                                                   + np.sin(ang)[..., None] * b[:, None, :])
        if kind == "straddle":  # one vertex in front of, one behind the near plane
            v[:, 0, 2] = eye[2] - (near - 0.6 * size)
            v[:, 1, 2] = eye[2] - (near + 0.6 * size)
        nrm = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
        nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-20)
        return v.astype(np.float32), nrm.astype(np.float32)

    def add_mesh(v, nrm, oid):
        nt = v.shape[0]
        pos = v.reshape(-1, 3)
        nn = np.repeat(nrm, 3, axis=0)
        col = np.repeat(rng.uniform(0.2, 1.0, (nt, 4)).astype(np.float32), 3, axis=0)
        col[:, 3] = 1.0
        uv = np.zeros((3 * nt, 2), np.float32)
        verts = _pack(pos, nn, col, uv)
        idx = np.arange(3 * nt, dtype=np.uint32)
        m, r = _mat_rand(rng)
        sc.meshes.append(Mesh(verts, idx, oid, mat_identity(), m, r))

    oid = 1
    counts = {"plain": int(n_tris * 0.60), "pair": int(n_tris * 0.10),
              "straddle": int(n_tris * 0.10), "outside": int(n_tris * 0.05)}
    for kind in ("plain", "straddle", "outside"):
        v, nrm = tris(counts[kind], kind)
        for s0 in range(0, v.shape[0], tris_per_mesh):
            add_mesh(v[s0:s0 + tris_per_mesh], nrm[s0:s0 + tris_per_mesh], oid)
            oid += 1
    v, nrm = tris(counts["pair"], "plain")          # coplanar pairs: same triangles twice
    for s0 in range(0, v.shape[0], tris_per_mesh):
        for _ in range(2):
            add_mesh(v[s0:s0 + tris_per_mesh], nrm[s0:s0 + tris_per_mesh], oid)
            oid += 1
    # joint-skinned tubes: 64 joints along each tube, 4 influences per vertex
    skinned = n_tris - sum(counts.values()) - counts["pair"]
    seg, ring = 64, 16
    per_tube = 2 * seg * ring
    for _ in range(max(1, skinned // per_tube)):
        z = np.linspace(0.0, 1.0, seg + 1)
        a = np.linspace(0.0, 2 * math.pi, ring, endpoint=False)
        Z, A = np.meshgrid(z, a, indexing="ij")
        rad = 0.15
        pos = np.stack([rad * np.cos(A), rad * np.sin(A), Z * 4.0], -1).reshape(-1, 3)
        nrm = np.stack([np.cos(A), np.sin(A), np.zeros_like(A)], -1).reshape(-1, 3)
        col = np.tile(rng.uniform(0.2, 1.0, 4).astype(np.float32), (pos.shape[0], 1))
        col[:, 3] = 1.0
        verts = _pack(pos.astype(np.float32), nrm.astype(np.float32), col,
                      np.zeros((pos.shape[0], 2), np.float32))
        jpos = np.clip((Z.reshape(-1) * 63.0), 0, 63)
        j0 = np.floor(jpos).astype(np.int64)
        joints = np.clip(np.stack([j0 - 1, j0, j0 + 1, j0 + 2], 1), 0, 63)
        w = rng.uniform(0.05, 1.0, (pos.shape[0], 4)).astype(np.float32)
        w /= w.sum(1, keepdims=True)
        mats = []
        base = rng.uniform(-3, 3, 3) + np.array([0.0, 0.0, -5.0])
        for j in range(64):
            ang = 0.6 * math.sin(j / 64.0 * math.pi * rng.uniform(0.5, 2.0))
            rot = np.array([[math.cos(ang), -math.sin(ang), 0], [math.sin(ang), math.cos(ang), 0],
                            [0, 0, 1]])
            mats.append(mat_trs(base + np.array([0.0, 0.02 * j, 0.0]), rot, (1.0, 1.0, 1.0)))
        verts = skin_vertices(verts, joints, w, np.asarray(mats, np.float32))
        idx = []
        for s_ in range(seg):
            for r_ in range(ring):
                i0 = s_ * ring + r_
                i1 = s_ * ring + (r_ + 1) % ring
                i2 = i0 + ring
                i3 = i1 + ring
                idx += [i0, i1, i3, i0, i3, i2]
        m, r = _mat_rand(rng)
        sc.meshes.append(Mesh(verts, np.asarray(idx, np.uint32), oid, mat_identity(), m, r))
        oid += 1
    return sc


BLEND_OPAQUE, BLEND_ALPHA, BLEND_ADDITIVE, BLEND_MULTIPLY = 0, 1, 2, 3


def effective_blend(m: Mesh) -> int:
    """The mesh's blend mode as the core holds it: mop_mesh_set_opacity
    promotes an opaque mesh to alpha blending below opacity 1
    (reference viewport.c:1815-1829)."""
    if m.blend_mode:
        return m.blend_mode
    return BLEND_ALPHA if m.opacity < 1.0 else BLEND_OPAQUE


def draw_order(scene: Scene, eye) -> List[int]:
    """Mesh indices in the core's draw order (viewport.c:2449-2553): opaque
    meshes in scene order, then blended meshes back to front by the float32
    squared distance of their translation to the eye (the core's insertion
    sort: farthest first, ties keep scene order); IDs in the hidden range are
    not drawn."""
    shown = [k for k, m in enumerate(scene.meshes)
             if m.object_id < HIDDEN_ID_FLOOR and m.object_id != GRID_ID]
    opaque = [k for k in shown if effective_blend(scene.meshes[k]) == BLEND_OPAQUE]
    trans = [k for k in shown if effective_blend(scene.meshes[k]) != BLEND_OPAQUE]
    e = np.asarray(eye, np.float32)
    dist = []
    for k in trans:
        t = np.asarray(scene.meshes[k].transform, np.float32)
        dx, dy, dz = t[12] - e[0], t[13] - e[1], t[14] - e[2]
        dist.append(np.float32(np.float32(dx * dx + dy * dy) + dz * dz))
    idx = list(trans)
    for j in range(1, len(idx)):
        ki, kd = idx[j], dist[j]
        i = j - 1
        while i >= 0 and dist[i] < kd:
            idx[i + 1], dist[i + 1] = idx[i], dist[i]
            i -= 1
        idx[i + 1], dist[i + 1] = ki, kd
    return opaque + idx


def transparent_scene(seed: int = 12, width: int = 160, height: int = 120, ssaa: int = 1,
                      env: int = 0) -> Scene:
    """small_scene plus overlapping blended meshes: alpha (opacity 0.2-0.9),
    additive and multiply spheres and quads in front of and behind the opaque
    ones, so blended fragments stack, pass and fail the depth test, and write
    depth and IDs when their alpha exceeds 0.5."""
    sc = small_scene(seed=seed, width=width, height=height, ssaa=ssaa, env=env)
    rng = np.random.default_rng(seed + 100)
    oid = max(m.object_id for m in sc.meshes) + 1
    modes = [BLEND_OPAQUE, BLEND_OPAQUE, BLEND_ALPHA, BLEND_ADDITIVE, BLEND_MULTIPLY, BLEND_OPAQUE]
    for k, mode in enumerate(modes):
        v, i = uv_sphere(24, 12, float(rng.uniform(0.4, 0.9)), _color(rng))
        t = rng.uniform(-1.2, 1.2, 3)
        m = mat_trs(t, random_rotation(rng), (1.0, 1.0, 1.0))
        mt, r = _mat_rand(rng)
        op = float(rng.uniform(0.2, 0.9)) if mode in (BLEND_OPAQUE, BLEND_ALPHA) else \
            float(rng.uniform(0.3, 1.0))
        sc.meshes.append(Mesh(v, i, oid, m, mt, r, opacity=op, blend_mode=mode))
        oid += 1
    return sc


def deep_transparent_scene(seed: int = 64, width: int = 160, height: int = 120, ssaa: int = 1,
                           layers: int = 64) -> Scene:
    """small_scene with `layers` blended quads stacked along z in front of
    the camera (alpha, additive, multiply and alpha-promoted opaque, opacity
    0.05-0.7), so the middle samples receive more blended fragments than a
    sample's sorted register list holds (48): the scratch heapsort orders
    them."""
    sc = small_scene(seed=seed, width=width, height=height, ssaa=ssaa)
    rng = np.random.default_rng(seed + 200)
    oid = max(m.object_id for m in sc.meshes) + 1
    modes = [BLEND_ALPHA, BLEND_ADDITIVE, BLEND_MULTIPLY, BLEND_OPAQUE]
    for k in range(layers):
        j = rng.uniform(-0.15, 0.15, 4)
        v, i = _quad(-1.3 + j[0], -0.9 + j[1], 1.3 + j[2], 0.9 + j[3], 0.0, _color(rng))
        z = -1.5 + 3.0 * k / max(1, layers - 1)
        m = mat_trs((float(rng.uniform(-0.1, 0.1)), 1.0, z), np.eye(3), (1.0, 1.0, 1.0))
        sc.meshes.append(Mesh(v, i, oid, m, 0.0, 0.5, opacity=float(rng.uniform(0.05, 0.7)),
                              blend_mode=modes[k % 4]))
        oid += 1
    return sc


def wireframe_scene(seed: int = 110, width: int = 160, height: int = 120, ssaa: int = 1,
                    lights: str = "mixed") -> Scene:
    """small_scene in MOP_RENDER_WIREFRAME, plus an ID-0 quad (drawn filled:
    the core keeps ID 0 solid) and a long thin triangle crossing the view
    (steep and shallow edges, sub-pixel ends)."""
    sc = small_scene(seed=seed, width=width, height=height, ssaa=ssaa, lights=lights)
    v, i = _quad(-3.0, 0.2, -1.0, 1.4, 0.5, (0.9, 0.4, 0.2, 1.0))
    sc.meshes.append(Mesh(v, i, 0, mat_identity()))
    pos = np.array([[-4.0, 0.3, -1.0], [4.5, 2.6, 0.4], [-3.7, 0.45, -0.9]], np.float32)
    nrm = np.tile(np.array([0.0, 1.0, 0.0], np.float32), (3, 1))
    col = np.tile(np.array([0.3, 0.8, 1.0, 1.0], np.float32), (3, 1))
    uv = np.zeros((3, 2), np.float32)
    oid = max(m.object_id for m in sc.meshes) + 1
    sc.meshes.append(Mesh(_pack(pos, nrm, col, uv), np.array([0, 1, 2, 0, 2, 1], np.uint32), oid,
                          mat_identity()))
    return dataclasses.replace(sc, wireframe=True)


def fuzz_scene(seed: int) -> Scene:
    """A seeded random frame for parity sweeps: 1-3 SSAA, random camera;
    a ground plane plus 3-8 meshes drawn from spheres, tori and raw
    triangle soups (degenerate, sliver, huge, behind the eye, straddling the
    near plane, outside the frustum), random materials, opacities and blend
    modes, some editor-chrome IDs; 0-5 lights of every type (some inactive,
    some range-limited); smooth or flat shading, sometimes wireframe; random
    post effects incl. fog and vignette."""
    rng = np.random.default_rng(10_000 + seed)
    w = int(rng.integers(40, 130))
    h = int(rng.integers(30, 100))
    ssaa = int(rng.integers(1, 4))
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    eye = tuple(float(x) for x in d * rng.uniform(3.0, 9.0))
    target = tuple(float(x) for x in rng.uniform(-0.5, 0.5, 3))
    sc = Scene(f"fuzz{seed}", w, h, ssaa, eye=eye, target=target,
               fov_deg=float(rng.uniform(30.0, 90.0)), near=float(rng.uniform(0.05, 0.5)),
               far=float(rng.uniform(20.0, 100.0)), sun_dir=(0.3, 0.8, 0.4))
    n_lights = int(rng.integers(0, 6))
    for k in range(n_lights):
        t = int(rng.integers(0, 3))
        p = tuple(float(x) for x in rng.uniform(-4, 4, 3))
        dr = rng.normal(size=3)
        dr /= np.linalg.norm(dr)
        inner = float(rng.uniform(0.8, 0.99))
        sc.lights.append(Light(t, position=p, direction=tuple(float(x) for x in dr),
                               color=(*[float(x) for x in rng.uniform(0.3, 1.0, 3)], 1.0),
                               intensity=float(rng.uniform(0.5, 30.0)),
                               range=float(rng.uniform(2.0, 10.0)) if rng.random() < 0.3 else 0.0,
                               spot_inner_cos=inner, spot_outer_cos=inner - float(rng.uniform(0.0, 0.2)),
                               active=bool(rng.random() < 0.85)))
    if rng.random() < 0.5:
        sc.textures.append(value_noise_texture(rng, 32, 4))
    v, i = ground_plane(float(rng.uniform(4.0, 20.0)), _color(rng))
    sc.meshes.append(Mesh(v, i, 1, mat_identity(), *_mat_rand(rng)))
    oid = 2
    for n in range(int(rng.integers(3, 9))):
        kind = int(rng.integers(0, 4))
        c = _color(rng)
        if kind == 0:
            v, i = uv_sphere(int(rng.integers(6, 20)), int(rng.integers(4, 10)),
                             float(rng.uniform(0.2, 1.2)), c)
        elif kind == 1:
            v, i = torus(int(rng.integers(8, 24)), int(rng.integers(4, 12)), 0.8, 0.25, c)
        else:  # triangle soup with awkward cases
            nt = int(rng.integers(4, 40))
            pos = rng.uniform(-2.5, 2.5, (nt * 3, 3)).astype(np.float32)
            for t in range(nt):
                r = rng.random()
                if r < 0.1:  # degenerate: repeated vertex
                    pos[3 * t + 2] = pos[3 * t]
                elif r < 0.2:  # sliver
                    pos[3 * t + 2] = pos[3 * t] + (pos[3 * t + 1] - pos[3 * t]) * 0.5 + 1e-4
                elif r < 0.3:  # huge
                    pos[3 * t:3 * t + 3] *= 40.0
                elif r < 0.4:  # through the eye / near plane
                    pos[3 * t] = np.asarray(eye, np.float32) * float(rng.uniform(0.8, 1.2))
            nrm = rng.normal(size=(nt * 3, 3)).astype(np.float32)
            nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
            col = np.concatenate([rng.uniform(0, 1, (nt * 3, 3)), np.ones((nt * 3, 1))], 1)
            uv = rng.uniform(0, 1, (nt * 3, 2))
            v = _pack(pos, nrm, col.astype(np.float32), uv.astype(np.float32))
            i = np.arange(nt * 3, dtype=np.uint32)
        t = rng.uniform(-2.0, 2.0, 3)
        s_ = float(rng.uniform(0.5, 1.5))
        m = mat_trs(t, random_rotation(rng), (s_, s_, s_))
        mt, rough = _mat_rand(rng)
        r = rng.random()
        op, bm = 1.0, BLEND_OPAQUE
        if r < 0.2:
            op, bm = float(rng.uniform(0.1, 0.9)), BLEND_ALPHA
        elif r < 0.3:
            op, bm = float(rng.uniform(0.3, 1.0)), BLEND_ADDITIVE
        elif r < 0.4:
            op, bm = float(rng.uniform(0.3, 1.0)), BLEND_MULTIPLY
        mid = CHROME_ID_FLOOR + 32 + n if rng.random() < 0.1 else oid
        oid += 1
        tex = 0 if (sc.textures and rng.random() < 0.5) else -1
        sc.meshes.append(Mesh(v, i, mid, m, mt, rough, texture=tex, opacity=op, blend_mode=bm))
    post = DEFAULT_POST
    if rng.random() < 0.3:
        post |= POST_TONEMAP
    if rng.random() < 0.2:
        post |= POST_VIGNETTE
    fog = None
    if rng.random() < 0.2:
        post |= POST_FOG
        fog = ((*[float(x) for x in rng.uniform(0, 1, 3)], 1.0), float(rng.uniform(0.8, 0.95)),
               float(rng.uniform(0.95, 1.0)))
    return dataclasses.replace(sc, smooth=bool(rng.random() < 0.75),
                               wireframe=seed % 6 == 5 or bool(rng.random() < 0.1),
                               post_effects=post, fog=fog)


def instanced_scene(seed: int = 70, width: int = 192, height: int = 144, ssaa: int = 1,
                    n_instances: int = 96, transparent: bool = False, env: int = 0,
                    zero_id: bool = False) -> Scene:
    """small_scene (or transparent_scene) plus an instanced icosphere: n_instances
    copies with one object ID scattered through the opaque meshes, so instances
    overlap each other and the scene.  The core draws them after the transparent
    pass with the depth write off (each instance's depth is undone after it), so
    a later instance behind an earlier one, but in front of the scene, replaces
    its colour and ID.  zero_id adds 64 instanced tori with object ID 0 (back
    faces not culled, resolved as background)."""
    if transparent:
        sc = transparent_scene(seed=seed, width=width, height=height, ssaa=ssaa, env=env)
    else:
        sc = small_scene(seed=seed, width=width, height=height, ssaa=ssaa, env=env)
    sc.name = f"instanced{seed}"
    rng = np.random.default_rng(seed + 300)

    def scatter(n, smin, smax):
        out = np.zeros((n, 16), np.float32)
        for k in range(n):
            t = rng.uniform(-2.8, 2.8, 3)
            t[1] = float(rng.uniform(0.1, 1.8))
            s = float(rng.uniform(smin, smax))
            out[k] = mat_trs(t, random_rotation(rng), (s, s, s))
        return out

    v, i = icosphere(1, 0.3, _color(rng))
    sc.instanced.append(InstancedMesh(v, i, 100, scatter(n_instances, 0.5, 1.3)))
    if zero_id:
        v, i = torus(16, 8, 0.35, 0.12, _color(rng))
        sc.instanced.append(InstancedMesh(v, i, 0, scatter(64, 0.6, 1.4)))
    return sc


def bc_scene(seed: int = 90, width: int = 192, height: int = 144, ssaa: int = 1) -> Scene:
    """small_scene whose meshes sample block-compressed textures (BC1, BC3
    and BC5 of odd sizes, so the last row and column of blocks are clamped)
    besides an RGBA8 one: textures modulate vertex colours at the vertices."""
    sc = small_scene(seed=seed, width=width, height=height, ssaa=ssaa, n_meshes=8)
    sc.name = f"bc{seed}"
    rng = np.random.default_rng(seed + 700)
    sc.textures.append(bc_texture(rng, TEX_BC1, 61, 47))
    sc.textures.append(bc_texture(rng, TEX_BC3, 64, 64))
    sc.textures.append(bc_texture(rng, TEX_BC5, 33, 70))
    for k in range(1, len(sc.meshes)):
        sc.meshes[k].texture = k % 4
    return sc


SHADOW_MAP_SIZE = 1024          # MOP_SHADOW_MAP_SIZE, reference viewport.c:2286
CHROME_ID_FLOOR = 0xFFFD0000    # object IDs at or above it are editor chrome
HIDDEN_ID_FLOOR = 0xFFFE0000    # object IDs at or above it are not drawn by the scene passes
GRID_ID = 0xFFFD0001            # MOP_GRID_ID: drawn only by the chrome grid pass (viewport.c:122)


def is_chrome(object_id: int) -> bool:
    """EMIT_DRAW's chrome test (reference viewport.c:2035-2076): a chrome draw
    has the depth test and back-face culling off, no light list (the legacy
    single-light path) and ambient 1."""
    return object_id >= CHROME_ID_FLOOR


def chrome_scene(seed: int = 80, width: int = 192, height: int = 144, ssaa: int = 1) -> Scene:
    """small_scene with three meshes in the editor-chrome ID range among its
    opaque meshes: they draw over what came before them (depth test off) and
    write depth that later meshes test against; one mesh in the hidden range
    and one with the grid's ID are skipped by the scene passes."""
    sc = small_scene(seed=seed, width=width, height=height, ssaa=ssaa, n_meshes=7)
    sc.name = f"chrome{seed}"
    rng = np.random.default_rng(seed + 500)
    chrome = []
    for k in range(3):
        v, i = icosphere(2, float(rng.uniform(0.4, 0.7)), _color(rng)) if k != 1 else \
            torus(24, 12, 0.8, 0.2, _color(rng))
        t = rng.uniform(-1.5, 1.5, 3)
        t[1] = float(rng.uniform(0.4, 1.4))
        chrome.append(Mesh(v, i, CHROME_ID_FLOOR + 16 + k, mat_trs(t, random_rotation(rng),
                                                                   (1.0, 1.0, 1.0))))
    v, i = icosphere(1, 2.0, _color(rng))
    hidden = Mesh(v, i, HIDDEN_ID_FLOOR + 5, mat_identity())
    # chrome meshes among the opaque ones and last; the hidden one after the first, the
    # grid-ID one after the first chrome mesh
    sc.meshes.insert(1, hidden)
    v, i = icosphere(1, 1.5, _color(rng))
    sc.meshes.insert(3, Mesh(v, i, GRID_ID, mat_identity()))
    sc.meshes.insert(2, chrome[0])
    sc.meshes.insert(5, chrome[1])
    sc.meshes.append(chrome[2])
    return sc


def shadow_light(scene: Scene):
    """The light pass_shadow renders from: the first active directional light
    with cast_shadows (reference viewport.c:2293-2300), or None."""
    for l in scene.lights:
        if l.active and l.type == LIGHT_DIRECTIONAL and l.cast_shadows:
            return l
    return None


def shadow_casters(scene: Scene) -> List[int]:
    """Mesh indices pass_shadow rasterises, in mesh order: active opaque
    meshes below the chrome IDs (viewport.c:2310-2315, 2405-2410)."""
    return [k for k, m in enumerate(scene.meshes)
            if m.object_id < CHROME_ID_FLOOR and effective_blend(m) == BLEND_OPAQUE]


def shadow_scene(seed: int = 31, width: int = 192, height: int = 144, ssaa: int = 1,
                 env: int = 0, transparent: bool = False) -> Scene:
    """small_scene (or transparent_scene) with its directional light casting
    shadows onto the ground plane, plus a second directional light that does
    not cast: the bound map shadows every directional light's diffuse and
    specular terms (reference rasterizer.c:1580-1583, 1677-1680, 1802-1805)."""
    if transparent:
        sc = transparent_scene(seed=seed, width=width, height=height, ssaa=ssaa, env=env)
    else:
        sc = small_scene(seed=seed, width=width, height=height, ssaa=ssaa, env=env)
    sc.name = f"shadow{seed}"
    sc.lights[0].cast_shadows = True
    sc.lights.append(Light(LIGHT_DIRECTIONAL, direction=(0.5, -0.8, 0.2), intensity=0.8,
                           color=(0.9, 0.9, 1.0, 1.0)))
    return sc


@dataclasses.dataclass
class View:
    """One viewport of a batch: presented size, SSAA factor and camera."""
    width: int
    height: int
    ssaa: int
    eye: Tuple[float, float, float]
    target: Tuple[float, float, float]
    up: Tuple[float, float, float] = (0.0, 1.0, 0.0)
    fov_deg: float = 50.0
    near: float = 0.5
    far: float = 200.0
    clear: Tuple[float, float, float, float] = (0.12, 0.13, 0.16, 1.0)

    @property
    def samples(self) -> int:
        return self.width * self.ssaa * self.height * self.ssaa

    @property
    def pixels(self) -> int:
        return self.width * self.height


def batch_views(scene: Scene, n: int = 64, seed: int = 4, min_px: int = 128 * 128,
                max_px: int = 1920 * 1080, radius=(15.0, 40.0)) -> List[View]:
    """Viewports of the batched workload over `scene`: presented pixel counts
    log-uniform in [min_px, max_px], aspect ratio log-uniform in [0.5, 2],
    ssaa 1 or 2, cameras on a sphere of radius U[radius] around the origin
    looking at a random instance's position."""
    rng = np.random.default_rng(seed)
    targets = [tuple(float(x) for x in m.transform[12:15]) for m in scene.meshes] or [(0.0, 0.0, 0.0)]
    views = []
    for _ in range(n):
        px = math.exp(rng.uniform(math.log(min_px), math.log(max_px)))
        aspect = math.exp(rng.uniform(math.log(0.5), math.log(2.0)))
        w = max(16, int(round(math.sqrt(px * aspect))))
        h = max(16, int(round(px / w)))
        ssaa = int(rng.integers(1, 3))
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        eye = tuple(float(x) for x in d * rng.uniform(*radius))
        tgt = targets[int(rng.integers(0, len(targets)))]
        views.append(View(w, h, ssaa, eye, tgt, clear=scene.clear))
    return views


def scene_for_view(scene: Scene, v: View) -> Scene:
    """The single-viewport scene a batch viewport corresponds to."""
    return dataclasses.replace(scene, width=v.width, height=v.height, ssaa=v.ssaa, eye=v.eye,
                               target=v.target, up=v.up, fov_deg=v.fov_deg, near=v.near,
                               far=v.far, clear=v.clear)


def procedural_ibl(sun_dir=(0.4, 0.8, 0.35), irr_size=(64, 32), pf_size=(128, 64), levels=5,
                   brdf_size=256, rotation=0.0, intensity=1.0) -> dict:
    """Seedless procedural sky and derived IBL maps with the reference's map
    sizes (irradiance 64x32, prefiltered 128x64 x 5 levels concatenated, BRDF
    LUT 256^2, all RGBA32F; reference src/core/environment.c:111-484).

    The content is a smooth gradient sky with a sun lobe, blurred per level;
    the BRDF LUT is a smooth split-sum-shaped table.  The frame path's work
    (lookups, bilinear filtering, LUT fetches) does not depend on the values,
    so the benchmark uses these maps; parity tests use the maps the reference
    library itself precomputes."""
    sd = np.asarray(sun_dir, np.float64)
    sd /= np.linalg.norm(sd)

    def sky(w, h, blur):
        u = (np.arange(w) + 0.5) / w
        v = (np.arange(h) + 0.5) / h
        phi = (u - 0.5) * 2.0 * math.pi
        th = (v - 0.5) * math.pi
        P, T = np.meshgrid(phi, th)
        d = np.stack([np.cos(T) * np.cos(P), np.sin(T), np.cos(T) * np.sin(P)], -1)
        up = np.clip(d[..., 1], -1.0, 1.0)
        base = np.stack([0.35 + 0.25 * up, 0.45 + 0.25 * up, 0.65 + 0.3 * up], -1)
        base = np.where(up[..., None] < 0, np.array([0.18, 0.16, 0.14]), base)
        cosang = np.clip((d * sd).sum(-1), -1.0, 1.0)
        sharp = 400.0 / (1.0 + 60.0 * blur)
        sun = (6.0 / (1.0 + 20.0 * blur)) * np.exp(sharp * (cosang - 1.0))
        rgb = base * (1.0 - 0.5 * blur) + sun[..., None] * np.array([1.0, 0.95, 0.85])
        out = np.ones((h, w, 4), np.float32)
        out[..., :3] = rgb
        return out

    iw, ih = irr_size
    irr = sky(iw, ih, 1.0)
    pw, ph = pf_size
    pf = []
    for l in range(levels):
        lw, lh = max(1, pw >> l), max(1, ph >> l)
        pf.append(sky(lw, lh, l / max(1, levels - 1)).reshape(-1))
    ndv = (np.arange(brdf_size) + 0.5) / brdf_size
    rough = (np.arange(brdf_size) + 0.5) / brdf_size
    N, R = np.meshgrid(ndv, rough)
    scale = np.clip(1.0 - 0.6 * R * (1.0 - N) - 0.3 * (1.0 - N) ** 5, 0.0, 1.0)
    bias = np.clip(0.08 * (1.0 - N) ** 5 * (1.0 - R) + 0.02 * R, 0.0, 1.0)
    lut = np.zeros((brdf_size, brdf_size, 4), np.float32)
    lut[..., 0] = scale
    lut[..., 1] = bias
    lut[..., 3] = 1.0
    return {"irr": irr.reshape(-1), "irr_w": iw, "irr_h": ih,
            "pf": np.concatenate(pf).astype(np.float32), "pf_w": pw, "pf_h": ph,
            "pf_levels": levels, "brdf": lut.reshape(-1), "brdf_size": brdf_size,
            "rotation": float(rotation), "intensity": float(intensity)}


def pick_points(scene: Scene, n: int = 1000, seed: int = 11) -> np.ndarray:
    rng = np.random.default_rng(seed)
    xy = np.empty((n, 2), np.int32)
    xy[:, 0] = rng.integers(0, scene.width, n)
    xy[:, 1] = rng.integers(0, scene.height, n)
    return xy
