"""Seeded synthetic scenes for the path-tracing workloads.

The reference renders hand-built analytic scenes plus glTF meshes
(main.cpp:53-345, cargarModelo.h); its assets are not used here.  These
generators build the same kinds of inputs -- analytic primitives, triangle
meshes with per-vertex normals, point lights -- as `Primitiva` / `LuzPuntual`
/ `Camara` arrays, deterministically from a seed:

* ``box_icosphere``   12-triangle box + displaced icosphere (subdiv 6, 81,920
                      triangles), one light: 512x512 plain path tracing.
* ``spheres_terrain`` 16 displaced icospheres (subdiv 5) + fractal terrain
                      heightfield, ~1.0M triangles, two lights: 1920x1080.
* ``tiny``            small variants of both for parity tests.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .structs import CAMARA, ESFERA, LUZ, PLANO, PRIMITIVA, TRIANGULO, set_sphere_radius


@dataclass
class Scene:
    prims: np.ndarray                 # analytic primitives (PRIMITIVA), tested by brute force
    mesh: np.ndarray                  # TRIANGULO primitives traversed through the CWBVH
    lights: np.ndarray                # LUZ
    camera: np.ndarray                # CAMARA, shape (1,)
    width: int
    height: int
    bounds: tuple = field(default=((-1, -1, -1), (1, 1, 1)))   # NRC scene bounds (min, max)
    name: str = ""

    @property
    def n_tris(self) -> int:
        return len(self.mesh)


# ---------------------------------------------------------------- camera
def make_camera(pos, look_at, up=(0.0, 1.0, 0.0), width=512, height=512, fov_deg=45.0, focal=1.0) -> np.ndarray:
    """Camara built like camara.h:29-40 (orthonormalised frame) with the plane
    size of RenderKernel.cu:70-74 (vertical FOV, aspect W/H)."""
    p = np.asarray(pos, np.float64)
    f = np.asarray(look_at, np.float64) - p
    f /= np.linalg.norm(f)
    a = np.asarray(up, np.float64)
    a /= np.linalg.norm(a)
    left = np.cross(f, a)
    left /= np.linalg.norm(left)
    a = np.cross(left, f)
    a /= np.linalg.norm(a)
    fov = np.float32(fov_deg * math.pi / 180.0)
    alto = np.float32(2.0) * np.float32(focal) * np.float32(math.tan(fov / np.float32(2.0)))
    ancho = alto * (np.float32(width) / np.float32(height))
    cam = np.zeros(1, CAMARA)
    for name, v in (("posicion", p), ("frente", f), ("arriba", a), ("izquierda", left)):
        cam[name]["x"], cam[name]["y"], cam[name]["z"] = v
    cam["ancho_plano"], cam["alto_plano"], cam["distancia_focal"] = ancho, alto, focal
    return cam


def orbit_camera(center, radius, height, angle_deg, width, height_px, look_y=None) -> np.ndarray:
    a = math.radians(angle_deg)
    pos = (center[0] + radius * math.sin(a), height, center[2] + radius * math.cos(a))
    look = (center[0], center[1] if look_y is None else look_y, center[2])
    return make_camera(pos, look, width=width, height=height_px)


# ---------------------------------------------------------------- noise
class ValueNoise:
    """Seeded lattice value noise with smoothstep trilinear interpolation."""

    def __init__(self, seed: int, size: int = 64):
        rng = np.random.default_rng(seed)
        self.size = size
        self.lat = rng.uniform(-1.0, 1.0, size=(size, size, size))

    def __call__(self, p: np.ndarray) -> np.ndarray:
        s = self.size
        f = np.floor(p)
        t = p - f
        t = t * t * (3.0 - 2.0 * t)
        i = f.astype(np.int64) % s
        j = (i + 1) % s
        out = 0.0
        for dx in (0, 1):
            ix = (j if dx else i)[:, 0]
            wx = t[:, 0] if dx else 1.0 - t[:, 0]
            for dy in (0, 1):
                iy = (j if dy else i)[:, 1]
                wy = t[:, 1] if dy else 1.0 - t[:, 1]
                for dz in (0, 1):
                    iz = (j if dz else i)[:, 2]
                    wz = t[:, 2] if dz else 1.0 - t[:, 2]
                    out = out + wx * wy * wz * self.lat[ix, iy, iz]
        return out


# ---------------------------------------------------------------- meshes
def icosphere(subdiv: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20 * 4**subdiv triangles (counter-clockwise outward)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    V = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
                  (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
                  (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], np.int64)
    for _ in range(subdiv):
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = V[uniq[:, 0]] + V[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(V)
        V = np.concatenate([V, mid])
        nf = len(F)
        ab = base + inv[:nf]
        bc = base + inv[nf:2 * nf]
        ca = base + inv[2 * nf:]
        a, b, c = F[:, 0], F[:, 1], F[:, 2]
        F = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)])
    return V, F


def vertex_normals(V: np.ndarray, F: np.ndarray) -> np.ndarray:
    fn = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    N = np.zeros_like(V)
    for k in range(3):
        np.add.at(N, F[:, k], fn)
    N /= np.maximum(np.linalg.norm(N, axis=1, keepdims=True), 1e-30)
    return N


def displaced_icosphere(subdiv: int, center, radius: float, amp: float, seed: int, freq: float = 3.0):
    V, F = icosphere(subdiv)
    noise = ValueNoise(seed)
    d = noise(V * freq + 16.0)
    V = V * (radius * (1.0 + amp * d))[:, None] + np.asarray(center, np.float64)
    return V, F


def terrain(n: int, x0: float, x1: float, z0: float, z1: float, y0: float, height: float, seed: int):
    """Fractal (5-octave value-noise fBm) heightfield, 2 * n * n triangles."""
    xs = np.linspace(x0, x1, n + 1)
    zs = np.linspace(z0, z1, n + 1)
    X, Z = np.meshgrid(xs, zs, indexing="xy")
    noise = ValueNoise(seed)
    pts = np.stack([X.reshape(-1), np.zeros(X.size), Z.reshape(-1)], 1)
    h = np.zeros(X.size)
    amp, freq = 1.0, 0.15
    for _ in range(5):
        h += amp * noise(pts * freq + np.array([3.0, 7.5, 11.0]))
        amp *= 0.5
        freq *= 2.0
    V = np.stack([X.reshape(-1), y0 + height * h, Z.reshape(-1)], 1)
    idx = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1)
    a = idx[:-1, :-1].reshape(-1)
    b = idx[:-1, 1:].reshape(-1)
    c = idx[1:, :-1].reshape(-1)
    d = idx[1:, 1:].reshape(-1)
    F = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)])
    return V, F


def mesh_prims(V: np.ndarray, F: np.ndarray, kd: np.ndarray, smooth: bool = True) -> np.ndarray:
    """TRIANGULO primitives with per-vertex normals (cargarModelo.h builds the
    same from assimp meshes) and per-triangle diffuse albedo `kd` (n, 3)."""
    n = len(F)
    P = np.zeros(n, PRIMITIVA)
    P["tipo"] = TRIANGULO
    P["indice_refraccion"] = 1.0
    d = P["difuso"]
    d["r"], d["g"], d["b"] = kd[:, 0], kd[:, 1], kd[:, 2]
    N = vertex_normals(V, F) if smooth else None
    u = np.empty((n, 18), np.float64)
    for k in range(3):
        u[:, 3 * k:3 * k + 3] = V[F[:, k]]
        if smooth:
            u[:, 9 + 3 * k:12 + 3 * k] = N[F[:, k]]
        else:
            fn = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
            u[:, 9 + 3 * k:12 + 3 * k] = fn / np.maximum(np.linalg.norm(fn, axis=1, keepdims=True), 1e-30)
    P["u"] = u
    return P


def box_prims(lo, hi, colors: dict) -> np.ndarray:
    """12 analytic triangles (flat, equal vertex normals) forming a closed box."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    c = {
        "left": ((x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0)),
        "right": ((x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (x1, y0, z1)),
        "floor": ((x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1)),
        "ceiling": ((x0, y1, z0), (x0, y1, z1), (x1, y1, z1), (x1, y1, z0)),
        "back": ((x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (x1, y0, z0)),
        "front": ((x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)),
    }
    out = np.zeros(12, PRIMITIVA)
    k = 0
    for face, q in c.items():
        q = np.asarray(q, np.float64)
        fn = np.cross(q[1] - q[0], q[2] - q[0])
        fn /= np.linalg.norm(fn)
        for tri in ((q[0], q[1], q[2]), (q[0], q[2], q[3])):
            out[k]["tipo"] = TRIANGULO
            out[k]["indice_refraccion"] = 1.0
            col = colors.get(face, (0.75, 0.75, 0.75))
            out[k]["difuso"] = tuple(np.float32(v) for v in col)
            u = np.concatenate([tri[0], tri[1], tri[2], fn, fn, fn])
            out[k]["u"] = u
            k += 1
    return out


def sphere_prim(center, radius, kd=(0, 0, 0), ks=(0, 0, 0), kt=(0, 0, 0), ior=1.0, emission=(0, 0, 0)) -> np.ndarray:
    p = np.zeros(1, PRIMITIVA)
    p["tipo"] = ESFERA
    p["difuso"] = kd
    p["especular"] = ks
    p["transmision"] = kt
    p["emision"] = emission
    p["indice_refraccion"] = ior
    u = np.zeros(18)
    u[:3] = center
    p["u"] = u
    set_sphere_radius(p, slice(None), [radius])
    return p


def plane_prim(normal, dist, kd=(0.75, 0.75, 0.75)) -> np.ndarray:
    p = np.zeros(1, PRIMITIVA)
    p["tipo"] = PLANO
    p["difuso"] = kd
    p["indice_refraccion"] = 1.0
    u = np.zeros(18)
    u[:3] = normal
    p["u"] = u
    set_sphere_radius(p, slice(None), [dist])
    return p


def lights(*items) -> np.ndarray:
    L = np.zeros(len(items), LUZ)
    for i, (pos, inten) in enumerate(items):
        L[i]["posicion"] = tuple(pos)
        L[i]["intensidad"] = tuple(np.float32(v) for v in inten)
    return L


def _mesh_bounds(*arrays):
    pts = np.concatenate([a["u"][:, :9].reshape(-1, 3) for a in arrays if len(a)])
    lo, hi = pts.min(0), pts.max(0)
    pad = 0.05 * (hi - lo)
    return tuple((lo - pad).tolist()), tuple((hi + pad).tolist())


# ---------------------------------------------------------------- workloads
def box_icosphere(width=512, height=512, subdiv=6, seed=1) -> Scene:
    """Displaced icosphere (amplitude 0.1, 20*4**subdiv triangles) inside a
    12-triangle box, one point light; the sphere's Lambertian albedo is drawn
    from U[0.2, 0.8] per colour channel."""
    rng = np.random.default_rng(seed)
    V, F = displaced_icosphere(subdiv, (0.0, -0.8, -0.6), 1.0, 0.1, seed)
    kd = np.repeat(rng.uniform(0.2, 0.8, size=(1, 3)), len(F), axis=0).astype(np.float32)
    mesh = mesh_prims(V, F, kd)
    box = box_prims((-2.6, -2.0, -4.0), (2.6, 2.4, 5.5), {"left": (0.7, 0.2, 0.2), "right": (0.2, 0.7, 0.2)})
    L = lights(((0.0, 1.9, 0.8), (25.0, 25.0, 25.0)))
    cam = make_camera((0.0, -0.75, 4.25), (0.0, -0.75, 0.0), width=width, height=height)
    return Scene(box, mesh, L, cam, width, height, bounds=((-2.6, -2.0, -4.0), (2.6, 2.4, 5.5)),
                 name=f"box_icosphere_s{subdiv}")


def spheres_terrain(width=1920, height=1080, subdiv=5, terrain_n=580, seed=7, angle_deg=0.0) -> Scene:
    """16 displaced icospheres (20*4**subdiv triangles each) on a fractal
    heightfield (2*terrain_n**2 triangles); ~1.0M triangles at the defaults.
    Two point lights; each object's Lambertian albedo is drawn from
    U[0.1, 0.9] per colour channel."""
    rng = np.random.default_rng(seed)
    Vs, Fs, kds = [], [], []
    Vt, Ft = terrain(terrain_n, -10.0, 10.0, -18.0, 2.0, -1.8, 0.9, seed + 1)
    Vs.append(Vt); Fs.append(Ft)
    kds.append(np.repeat(rng.uniform(0.1, 0.9, size=(1, 3)), len(Ft), axis=0))
    off = len(Vt)
    k = 0
    for gx in (-6.0, -2.0, 2.0, 6.0):
        for gz in (-14.0, -10.0, -6.0, -2.0):
            r = float(rng.uniform(0.7, 1.3))
            c = (gx + float(rng.uniform(-0.8, 0.8)), -0.6 + r * 0.6, gz + float(rng.uniform(-0.8, 0.8)))
            V, F = displaced_icosphere(subdiv, c, r, 0.1, seed + 100 + k)
            Vs.append(V); Fs.append(F + off)
            kds.append(np.repeat(rng.uniform(0.1, 0.9, size=(1, 3)), len(F), axis=0))
            off += len(V)
            k += 1
    V = np.concatenate(Vs)
    F = np.concatenate(Fs)
    kd = np.concatenate(kds).astype(np.float32)
    mesh = mesh_prims(V, F, kd)
    L = lights(((-5.0, 8.0, -4.0), (140.0, 140.0, 140.0)), ((6.0, 6.0, 1.0), (90.0, 80.0, 70.0)))
    cam = orbit_camera((0.0, -1.0, -7.0), 13.0, 2.8, angle_deg, width, height)
    return Scene(np.zeros(0, PRIMITIVA), mesh, L, cam, width, height, bounds=_mesh_bounds(mesh),
                 name=f"spheres_terrain_{len(F)}")


def sized_terrain_scene(target_tris: int, width: int, height: int, n_lights: int, seed: int) -> Scene:
    """The spheres-over-terrain layout at a chosen size: 16 displaced
    icospheres carry about a third of `target_tris` (subdivision picked to
    fit), the heightfield the rest; 1-4 point lights on a ring above the
    scene.  Used for the batched multi-scene workload."""
    rng = np.random.default_rng(seed)
    subdiv = 0
    while subdiv < 7 and 16 * 20 * 4 ** (subdiv + 1) <= target_tris // 3:
        subdiv += 1
    n_sph = 16 * 20 * 4 ** subdiv
    terrain_n = max(8, int(round(np.sqrt(max(target_tris - n_sph, 128) / 2.0))))
    s = spheres_terrain(width, height, subdiv=subdiv, terrain_n=terrain_n, seed=seed)
    items = []
    for k in range(n_lights):
        a = 2.0 * np.pi * (k + float(rng.uniform(0.0, 0.5))) / n_lights
        pos = (7.0 * np.cos(a), float(rng.uniform(5.0, 9.0)), -6.0 + 7.0 * np.sin(a))
        items.append((pos, tuple(float(x) for x in rng.uniform(60.0, 140.0, 3))))
    s.lights = lights(*items)
    s.name = f"sized_terrain_{len(s.mesh)}_{width}x{height}_L{n_lights}"
    return s


# The batched workload: 12 scenes from 10k to 2M triangles (log-spaced),
# 1-4 lights, 640x360 to 1920x1080.
BATCH_RESOLUTIONS = [(640, 360), (960, 540), (1280, 720), (1600, 900), (1920, 1080)]


def batch_scene(i: int, n: int = 12) -> Scene:
    tris = int(round(np.exp(np.log(1e4) + (np.log(2e6) - np.log(1e4)) * i / max(1, n - 1))))
    w, h = BATCH_RESOLUTIONS[(i * 7) % len(BATCH_RESOLUTIONS)]
    return sized_terrain_scene(tris, w, h, 1 + (i % 4), seed=1000 + 17 * i)


def tiny_box(width=64, height=64, subdiv=2, seed=3) -> Scene:
    s = box_icosphere(width, height, subdiv, seed)
    s.name = f"tiny_box_s{subdiv}"
    return s


def reference_room(width=64, height=64, subdiv=2, seed=5) -> Scene:
    """Analytic planes and spheres of every material kind (diffuse, specular,
    transmissive, emissive) around a small displaced mesh -- the primitive
    mix of the reference's hand-built scenes (main.cpp:53-161)."""
    rng = np.random.default_rng(seed)
    prims = np.concatenate([
        plane_prim((-1.0, 0.0, 0.0), -4.0, kd=(0.8, 0.4, 0.1)),
        plane_prim((0.0, -0.25, 0.0), -3.0, kd=(0.9, 0.9, 0.9)),
        plane_prim((0.0, 0.0, 1.0), -10.0, kd=(0.9, 0.9, 0.9)),
        plane_prim((0.0, 1.0, 0.0), -2.0, kd=(0.6, 0.6, 0.6)),
        sphere_prim((-1.6, -1.1, -3.2), 0.7, kd=(0.1, 0.1, 0.1), ks=(0.3, 0.3, 0.3)),
        sphere_prim((0.9, -0.5, -1.8), 0.4, ks=(0.04, 0.04, 0.04), kt=(0.9, 0.1, 0.1), ior=3.0),
        sphere_prim((0.1, -1.1, -2.3), 0.15, ks=(0.04, 0.04, 0.04), kt=(0.1, 0.8, 0.4), ior=1.5),
        sphere_prim((1.8, 1.0, -4.0), 0.3, emission=(6.0, 5.0, 4.0)),
    ])
    V, F = displaced_icosphere(subdiv, (-0.6, -1.3, -2.2), 0.6, 0.1, seed)
    kd = np.repeat(rng.uniform(0.2, 0.8, size=(1, 3)), len(F), axis=0).astype(np.float32)
    mesh = mesh_prims(V, F, kd)
    L = lights(((0.0, -0.23, -2.0), (70.0, 70.0, 70.0)))
    cam = make_camera((0.0, -0.75, 4.25), (0.0, -0.75, 0.0), width=width, height=height)
    return Scene(prims, mesh, L, cam, width, height, bounds=((-6.0, -4.0, -10.0), (6.0, 6.0, 2.0)),
                 name="reference_room")
