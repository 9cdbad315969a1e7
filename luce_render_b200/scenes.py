"""Seeded synthetic scenes of the benchmark's shapes (the reference builds its test scenes
from luce-geocore primitives, which are not available here, so these generators are this
package's own; their triangle counts and layouts follow the workloads' descriptions).

- :func:`cornell_box` -- 5 walls + 2 boxes = 34 triangles in the unit cube, open toward +z.
- :func:`cornell_rays` -- 256x256 pinhole primary rays from (0, 0, 3) looking down -z (fov
  40 deg) and 65,536 random rays (origins uniform in the cube, directions uniform on
  the sphere).
- :func:`furnace` -- a closed icosphere (level 5: 20,480 triangles, radius 1), Lambertian
  albedo 0.8 emitting 1, the camera at its centre.
- :func:`incoherent_scene` -- 1,048,576 triangles: 512 icospheres (level 3, 1,280 each)
  and 512 tori (48 x 8 segments, 768 each), randomly placed, scaled and rotated in a
  100-unit box, albedo U(0.2, 0.9), 4 rect lights and 1 distant light.
- :func:`batch_scenes` -- the batched workload's size distribution.
"""
from __future__ import annotations

import math

import numpy as np

from . import (LIGHT_DISTANT, LIGHT_RECT, MeshData, OpenPbr, camera, light, look_frame, placement)

# ---- primitives ----------------------------------------------------------------------------


def icosphere(level: int, radius: float = 1.0):
    """A subdivided icosahedron: points on the sphere, 20 * 4^level triangles wound
    counter-clockwise seen from outside."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                      [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    faces = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                      [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                      [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    for _ in range(level):
        edges = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        uniq, inverse = np.unique(key, axis=0, return_inverse=True)
        inverse = inverse.reshape(-1)
        mids = verts[uniq[:, 0]] + verts[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = len(verts)
        verts = np.concatenate([verts, mids])
        f = len(faces)
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        ab, bc, ca = base + inverse[:f], base + inverse[f:2 * f], base + inverse[2 * f:]
        faces = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1),
                                np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)])
    return (verts * radius).astype(np.float32), faces.astype(np.uint32), verts.astype(np.float32)


def torus(major: int, minor: int, big: float = 1.0, small: float = 0.35):
    """A torus around +y: major x minor quads, 2 triangles each; points, indices, normals."""
    u = np.arange(major) * (2 * math.pi / major)
    v = np.arange(minor) * (2 * math.pi / minor)
    U, V = np.meshgrid(u, v, indexing="ij")
    cx, cz = np.cos(U), np.sin(U)
    px = (big + small * np.cos(V)) * cx
    pz = (big + small * np.cos(V)) * cz
    py = small * np.sin(V)
    pts = np.stack([px, py, pz], -1).reshape(-1, 3)
    nrm = np.stack([np.cos(V) * cx, np.sin(V), np.cos(V) * cz], -1).reshape(-1, 3)
    i = np.arange(major)[:, None]
    j = np.arange(minor)[None, :]
    a = i * minor + j
    b = ((i + 1) % major) * minor + j
    c = ((i + 1) % major) * minor + (j + 1) % minor
    d = i * minor + (j + 1) % minor
    tris = np.concatenate([np.stack([a, d, c], -1).reshape(-1, 3), np.stack([a, c, b], -1).reshape(-1, 3)])
    return pts.astype(np.float32), tris.astype(np.uint32), nrm.astype(np.float32)


def box_mesh(lo, hi):
    """An axis-aligned box: 8 points, 12 triangles (6 polygons of 2), wound outward."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    p = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float32)
    quads = [[0, 3, 2, 1], [4, 5, 6, 7], [0, 1, 5, 4], [2, 3, 7, 6], [1, 2, 6, 5], [0, 4, 7, 3]]
    tris, faces = [], []
    for f, q in enumerate(quads):
        tris += [[q[0], q[1], q[2]], [q[0], q[2], q[3]]]
        faces += [f, f]
    return p, np.array(tris, np.uint32), np.array(faces, np.uint32)


def _quad(p0, p1, p2, p3):
    return np.array([p0, p1, p2, p3], np.float32), np.array([[0, 1, 2], [0, 2, 3]], np.uint32)


# ---- the Cornell box (34 triangles) ------------------------------------------------------

WHITE, RED, GREEN = (0.73, 0.73, 0.73), (0.65, 0.05, 0.05), (0.12, 0.45, 0.15)


def cornell_meshes(materials: bool = False) -> list[MeshData]:
    """5 walls (10 triangles) and 2 boxes (24) in [-0.5, 0.5]^3, open toward +z. With
    `materials`, walls and boxes name library materials 1 (white), 2 (red), 3 (green)."""
    h = 0.5
    walls = [
        (_quad((-h, -h, -h), (h, -h, -h), (h, -h, h), (-h, -h, h)), 1),   # floor, facing +y
        (_quad((-h, h, -h), (-h, h, h), (h, h, h), (h, h, -h)), 1),       # ceiling, facing -y
        (_quad((-h, -h, -h), (-h, h, -h), (h, h, -h), (h, -h, -h)), 1),   # back wall, facing +z
        (_quad((-h, -h, -h), (-h, -h, h), (-h, h, h), (-h, h, -h)), 2),   # left wall (red), facing +x
        (_quad((h, -h, -h), (h, h, -h), (h, h, h), (h, -h, h)), 3),       # right wall (green), facing -x
    ]
    meshes = []
    for (pts, tris), mat in walls:
        meshes.append(MeshData(pts, tris, faces=[0, 0], face_count=1,
                               face_materials=[mat] if materials else None))
    for lo, hi, rot, pos in [((-0.15, -0.15, -0.15), (0.15, 0.15, 0.15), -0.31, (0.17, -0.35, 0.1)),
                             ((-0.15, -0.3, -0.15), (0.15, 0.3, 0.15), 0.28, (-0.18, -0.2, -0.15))]:
        p, t, f = box_mesh(lo, hi)
        meshes.append(MeshData(p, t, faces=f, face_count=6, face_materials=[1] * 6 if materials else None,
                               transform=placement(pos, (0.0, rot, 0.0))))
    return meshes


def cornell_materials():
    return [OpenPbr.lambert(WHITE), OpenPbr.lambert(RED), OpenPbr.lambert(GREEN)]


def cornell_light(intensity: float = 17.0):
    """A 0.5 x 0.5 rect light just below the ceiling, shining down (radiance 17)."""
    return light(LIGHT_RECT, position=(0.0, 0.499, 0.0), rotation=(-0.5 * math.pi, 0.0, 0.0),
                 intensity=intensity, width=0.5, height=0.5, normalize=False, visible=True)


def cornell_camera():
    """A pinhole at (0, 0, 3) looking down -z with a 40 deg field of view (square film)."""
    return camera((0.0, 0.0, 3.0), (0.0, 0.0, 0.0), focal_length=18.0 / math.tan(math.radians(20.0)),
                  horizontal_aperture=36.0)


def cornell_frame(width: int = 256, height: int = 256):
    return look_frame((0.0, 0.0, 3.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), math.tan(math.radians(20.0)),
                      width, height)


def random_rays(count: int, seed: int = 0x5EED0000, lo=-0.5, hi=0.5) -> np.ndarray:
    """Rays with origins uniform in the cube and directions uniform on the sphere
    (z = 1 - 2u, phi = 2 pi v): count x 8 floats (origin, tmin 0, direction, tmax 3e38)."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(count, 3))
    u, v = rng.random(count), rng.random(count)
    z = 1.0 - 2.0 * u
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = 2.0 * math.pi * v
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    rays = np.zeros((count, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    rays[:, 7] = 3.0e38
    return rays


def frame_rays(frame, jitter=None) -> np.ndarray:
    """The pixel-centre rays of a frame, f32 as the probe kernel makes them."""
    b = frame.pack()
    w, h = int(b[11]), int(b[15])
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    fx, fy = (x + np.float32(0.5)).reshape(-1), (y + np.float32(0.5)).reshape(-1)
    film = (b[4:7][None, :] + fx[:, None] * b[8:11][None, :]) + fy[:, None] * b[12:15][None, :]
    rays = np.zeros((w * h, 8), np.float32)
    rays[:, 0:3] = b[0:3]
    rays[:, 4:7] = film
    rays[:, 7] = 3.0e38
    return rays


# ---- the furnace -------------------------------------------------------------------------


def furnace_meshes(level: int = 5, radius: float = 1.0):
    p, t, n = icosphere(level, radius)
    return [MeshData(p, t, normals=-n, face_materials=None)]


def furnace_material(albedo: float = 0.8, emission: float = 1.0):
    return OpenPbr.lambert((albedo,) * 3, emission=emission)


# ---- the incoherent 1M-triangle scene ---------------------------------------------------


def incoherent_scene(seed: int = 0xC0FFEE, spheres: int = 512, tori: int = 512, sphere_level: int = 3,
                     torus_segments=(48, 8), extent: float = 50.0):
    """Meshes, library materials, lights and a camera for the incoherent-traversal
    workload: 2^20 triangles at the defaults."""
    rng = np.random.default_rng(seed)
    sp, st, sn = icosphere(sphere_level)
    tp, tt, tn = torus(*torus_segments)
    kinds = np.array([0] * spheres + [1] * tori)
    rng.shuffle(kinds)
    meshes, materials = [], []
    for i, kind in enumerate(kinds):
        pos = rng.uniform(-extent, extent, 3)
        scale = rng.uniform(0.5, 3.0)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                      [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                      [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]]) * scale
        m = np.concatenate([R[:, 0], R[:, 1], R[:, 2], pos])
        albedo = float(rng.uniform(0.2, 0.9))
        materials.append(OpenPbr.lambert((albedo, albedo, albedo)))
        p, t, n = (sp, st, sn) if kind == 0 else (tp, tt, tn)
        meshes.append(MeshData(p, t, normals=n, face_materials=np.full(len(t), i + 1, np.uint32),
                               transform=m))
    lights = []
    for k in range(4):
        ang = k * 0.5 * math.pi
        lights.append(light(LIGHT_RECT, position=(30.0 * math.cos(ang), 70.0, 30.0 * math.sin(ang)),
                            rotation=(-0.5 * math.pi, 0.0, 0.0), intensity=30.0, width=20.0, height=20.0))
    lights.append(light(LIGHT_DISTANT, rotation=(-1.0, 0.4, 0.0), intensity=2.0, angle=0.53))
    cam = camera((0.0, 0.0, 130.0), (0.0, 0.0, 0.0), focal_length=30.0, horizontal_aperture=36.0)
    return meshes, materials, lights, cam


def incoherent_rays(count: int, seed: int = 0x1C0DE, extent: float = 50.0) -> np.ndarray:
    """Incoherent rays through the 1M-triangle scene: origins uniform in its box,
    directions uniform on the sphere."""
    return random_rays(count, seed, -extent, extent)


# ---- the batched workload's scenes -------------------------------------------------------


def batch_plan(count: int = 64, seed: int = 0xBA7C4):
    """Per scene: triangle target (log-normal, median 20k, clipped to [1k, 500k]), film
    side (128..1024) and spectral flag (half each)."""
    rng = np.random.default_rng(seed)
    tris = np.clip(np.exp(rng.normal(math.log(20000.0), 1.0, count)), 1000, 500000).astype(np.int64)
    sides = rng.choice([128, 256, 512, 1024], count)
    spectral = np.array([i % 2 == 0 for i in range(count)])
    rng.shuffle(spectral)
    return [dict(triangles=int(t), side=int(s), spectral=bool(sp)) for t, s, sp in zip(tris, sides, spectral)]


def scene_of_size(triangles: int, seed: int):
    """A scene of the incoherent generator with about `triangles` triangles (spheres
    and tori of 1,280 and 768 triangles)."""
    objects = max(1, int(round(triangles / 1024)))
    spheres = objects // 2
    tori = objects - spheres
    extent = 50.0 * (objects / 1024.0) ** (1.0 / 3.0)
    return incoherent_scene(seed=seed, spheres=spheres, tori=tori, extent=max(extent, 4.0))


def grid(size: float, divisions: int):
    """A size x size square of divisions x divisions quads in the xz plane at y = 0,
    facing +y, 2 triangles (one polygon) a quad."""
    n = divisions
    s = np.linspace(-0.5 * size, 0.5 * size, n + 1)
    X, Z = np.meshgrid(s, s, indexing="ij")
    pts = np.stack([X, np.zeros_like(X), Z], -1).reshape(-1, 3).astype(np.float32)
    i = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    a = i * (n + 1) + j
    b = (i + 1) * (n + 1) + j
    c = (i + 1) * (n + 1) + j + 1
    d = i * (n + 1) + j + 1
    tris = np.stack([np.stack([a, d, c], -1), np.stack([a, c, b], -1)], 2).reshape(-1, 3).astype(np.uint32)
    faces = np.repeat(np.arange(n * n), 2).astype(np.uint32)
    return pts, tris, faces


def cube(size: float = 1.0):
    """A cube centred at the origin: 8 points, 12 triangles, 6 polygons."""
    h = 0.5 * size
    return box_mesh((-h, -h, -h), (h, h, h))


def probe_test_scene():
    """The probe check's scene (tests/gpu/main.lucb:24-41 in spirit): a 24-segment sphere,
    a placed cube and a 12 x 12 floor of 6 divisions, with a perspective (35 mm) and an
    orthographic camera."""
    sp, st, sn = icosphere(2, 1.0)
    cp, ct, cf = cube(1.0)
    gp, gt, gf = grid(12.0, 6)
    meshes = [MeshData(sp, st, normals=sn),
              MeshData(cp, ct, faces=cf, face_count=6, transform=placement((2.0, 0.0, -1.0), (0.3, 0.6, 0.0))),
              MeshData(gp, gt, faces=gf, face_count=36, transform=placement((0.0, -1.0, 0.0)))]
    cams = [camera((0.5, 1.0, 6.0), (-0.15, 0.05, 0.0), focal_length=35.0, horizontal_aperture=36.0),
            camera((0.0, 0.0, 8.0), (-0.3, 0.2, 0.0), projection=1, focal_length=50.0, horizontal_aperture=60.0)]
    return meshes, cams


# ---- glossy materials --------------------------------------------------------------------


def openpbr(**fields) -> OpenPbr:
    """OpenPbr.standard with the named fields set (colors as 3-tuples)."""
    m = OpenPbr.standard()
    for name, value in fields.items():
        if isinstance(value, (tuple, list)):
            getattr(m, name)[:] = list(value)
        else:
            setattr(m, name, value)
    return m


def glossy_cornell(ball_level: int = 3):
    """The benchmark's layout: a Cornell box spanning x, z in [-1, 1] and y in [0, 2], open
    toward +z (white floor, ceiling and back, red and green side walls, a 0.6 x 0.6 rect
    light under the ceiling), holding a tall blue box under a clear coat, a smooth glass
    ball, a rough gold ball, a small white cube and an orange rough plastic ball. Returns
    (meshes, cameras, lights, materials); library materials 1..7 are white, red, green,
    blue coat, glass, gold, orange."""
    walls = [
        (_quad((-1, 0, -1), (1, 0, -1), (1, 0, 1), (-1, 0, 1)), 1),    # floor, facing +y
        (_quad((-1, 2, -1), (-1, 2, 1), (1, 2, 1), (1, 2, -1)), 1),    # ceiling, facing -y
        (_quad((-1, 0, -1), (-1, 2, -1), (1, 2, -1), (1, 0, -1)), 1),  # back, facing +z
        (_quad((-1, 0, -1), (-1, 0, 1), (-1, 2, 1), (-1, 2, -1)), 2),  # left (red), facing +x
        (_quad((1, 0, -1), (1, 2, -1), (1, 2, 1), (1, 0, 1)), 3),      # right (green), facing -x
    ]
    meshes = [MeshData(p, t, faces=[0, 0], face_count=1, face_materials=[m]) for (p, t), m in walls]
    for lo, hi, turn, at, material in [((-0.275, 0.0, -0.275), (0.275, 1.2, 0.275), 0.26, (-0.38, 0.0, -0.35), 4),
                                       ((-0.175, 0.0, -0.175), (0.175, 0.35, 0.175), -0.3, (0.7, 0.0, 0.72), 1)]:
        p, t, f = box_mesh(lo, hi)
        meshes.append(MeshData(p, t, faces=f, face_count=6, face_materials=[material] * 6,
                               transform=placement(at, (0.0, turn, 0.0))))
    for radius, at, material in [(0.36, (0.3, 0.36, 0.05), 5), (0.26, (-0.5, 0.26, 0.5), 6),
                                 (0.16, (0.0, 0.16, 0.62), 7)]:
        p, t, n = icosphere(ball_level, radius)
        meshes.append(MeshData(p, t, normals=n, faces=np.zeros(len(t), np.uint32), face_count=1,
                               face_materials=[material], transform=placement(at)))
    materials = [openpbr(base_color=(0.73, 0.73, 0.73), specular_weight=0.0),
                 openpbr(base_color=(0.63, 0.065, 0.05), specular_weight=0.0),
                 openpbr(base_color=(0.14, 0.45, 0.091), specular_weight=0.0),
                 openpbr(base_color=(0.08, 0.16, 0.55), coat_weight=1.0, coat_roughness=0.05, specular_roughness=0.5),
                 openpbr(transmission_weight=1.0, specular_roughness=0.0, base_color=(1.0, 1.0, 1.0)),
                 openpbr(base_color=(1.0, 0.77, 0.34), base_metalness=1.0, specular_roughness=0.35),
                 openpbr(base_color=(0.9, 0.35, 0.05), specular_roughness=0.45, base_diffuse_roughness=0.5)]
    lights = [light(LIGHT_RECT, position=(0.0, 1.998, 0.0), rotation=(-0.5 * math.pi, 0.0, 0.0), intensity=15.0,
                    width=0.6, height=0.6, normalize=False, visible=True)]
    cams = [camera((0.0, 1.0, 3.9), (0.0, 0.0, 0.0), focal_length=18.0 / math.tan(math.radians(20.0)),
                   horizontal_aperture=36.0)]
    return meshes, cams, lights, materials


def furnace_sphere(level: int = 4):
    """A unit icosphere (smooth normals) at the origin and a camera at (0, 1, 4) looking at
    its centre (50 mm on a 36 mm film), for furnaces under a uniform background."""
    p, t, n = icosphere(level, 1.0)
    cam = camera((0.0, 1.0, 4.0), (-math.atan2(1.0, 4.0), 0.0, 0.0), focal_length=50.0, horizontal_aperture=36.0)
    return [MeshData(p, t, normals=n)], [cam]


def caustic_scene(sun_angle: float = 8.0, glass_roughness: float = 0.15):
    """Light paths from afar: an 8 x 8 floor (32 triangles) under a sun of `sun_angle`
    degrees and a dim sky, holding a glass ball (radius 0.5, the caustic caster), a gold
    ball and a white cube; no emitters of the light tree, so every light path starts on
    the disk facing the sun. Returns (meshes, cameras, lights, materials, background);
    library materials 1..3 are the floor's white, glass and gold."""
    p, t, f = grid(8.0, 4)
    meshes = [MeshData(p, t, faces=f, face_count=int(f.max()) + 1, face_materials=[1] * (int(f.max()) + 1))]
    for radius, at, material in [(0.5, (0.0, 0.5, 0.0), 2), (0.35, (-1.1, 0.35, -0.6), 3)]:
        sp, st, sn = icosphere(3, radius)
        meshes.append(MeshData(sp, st, normals=sn, faces=np.zeros(len(st), np.uint32), face_count=1,
                               face_materials=[material], transform=placement(at)))
    bp, bt, bf = box_mesh((-0.3, 0.0, -0.3), (0.3, 0.6, 0.3))
    meshes.append(MeshData(bp, bt, faces=bf, face_count=6, face_materials=[1] * 6,
                           transform=placement((1.2, 0.0, -0.8), (0.0, 0.4, 0.0))))
    materials = [openpbr(base_color=(0.8, 0.8, 0.8), specular_weight=0.0),
                 openpbr(transmission_weight=1.0, specular_roughness=glass_roughness, base_color=(1.0, 1.0, 1.0)),
                 openpbr(base_color=(1.0, 0.77, 0.34), base_metalness=1.0, specular_roughness=0.25)]
    lights = [light(LIGHT_DISTANT, rotation=(-0.75, 0.5, 0.0), intensity=3.0, angle=sun_angle)]
    cams = [camera((0.0, 2.2, 4.0), (-math.atan2(1.8, 4.0), 0.0, 0.0), focal_length=35.0, horizontal_aperture=36.0)]
    return meshes, cams, lights, materials, (0.05, 0.07, 0.1)
