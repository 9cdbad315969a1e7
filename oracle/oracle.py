"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so): TEST INFRASTRUCTURE.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module, as the
checker and the CPU baseline; the product never does. Build with ``make -C oracle``.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        build()
    return C.CDLL(str(LIB_PATH))


lib = _load()

NODE_DTYPE = np.dtype([("lo", "<f4", 3), ("first", "<u4"), ("hi", "<f4", 3), ("count", "<u4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("triangle", "<u4"), ("u", "<f4"), ("v", "<f4")])


class Counts(C.Structure):
    _fields_ = [("interior", C.c_uint64), ("triangles", C.c_uint64), ("dropped", C.c_uint64)]


class OrFrame(C.Structure):
    _fields_ = [("position", C.c_double * 3), ("corner", C.c_double * 3), ("du", C.c_double * 3),
                ("dv", C.c_double * 3), ("forward", C.c_double * 3), ("orthographic", C.c_int),
                ("width", C.c_uint32), ("height", C.c_uint32), ("lens_radius", C.c_double),
                ("focus_distance", C.c_double)]

    def pack(self) -> np.ndarray:
        """RayFrame.pack (camera.lucb:41-47): the 16 floats the kernels read."""
        return frame_pack(self)


class OrMesh(C.Structure):
    _fields_ = [("positions", C.POINTER(C.c_float)), ("point_count", C.c_uint64),
                ("indices", C.POINTER(C.c_uint32)), ("triangle_count", C.c_uint64),
                ("faces", C.POINTER(C.c_uint32)), ("face_count", C.c_uint32),
                ("normals", C.POINTER(C.c_float)), ("normals_per_corner", C.c_int),
                ("face_materials", C.POINTER(C.c_uint32)), ("transform", C.c_double * 12)]


class OrLight(C.Structure):
    _fields_ = [("matrix", C.c_double * 12), ("shape", C.c_int), ("color", C.c_double * 3),
                ("intensity", C.c_double), ("exposure", C.c_double), ("temperature", C.c_double),
                ("width", C.c_double), ("height", C.c_double), ("radius", C.c_double), ("angle", C.c_double),
                ("normalize", C.c_int), ("visible", C.c_int), ("image", C.POINTER(C.c_float)),
                ("image_width", C.c_uint32), ("image_height", C.c_uint32)]


class OrMaterial(C.Structure):
    _fields_ = [("base_weight", C.c_double), ("base_color", C.c_double * 3), ("base_metalness", C.c_double),
                ("base_diffuse_roughness", C.c_double), ("specular_weight", C.c_double),
                ("specular_color", C.c_double * 3), ("specular_roughness", C.c_double),
                ("specular_roughness_anisotropy", C.c_double), ("specular_ior", C.c_double),
                ("transmission_weight", C.c_double), ("transmission_color", C.c_double * 3),
                ("coat_weight", C.c_double), ("coat_color", C.c_double * 3), ("coat_roughness", C.c_double),
                ("coat_roughness_anisotropy", C.c_double), ("coat_ior", C.c_double),
                ("coat_darkening", C.c_double), ("emission_luminance", C.c_double),
                ("emission_color", C.c_double * 3), ("geometry_opacity", C.c_double),
                ("geometry_thin_walled", C.c_int), ("transmission_dispersion_scale", C.c_double),
                ("transmission_dispersion_abbe_number", C.c_double)]


class OrTree(C.Structure):
    _fields_ = [("nodes", C.POINTER(C.c_float)), ("links", C.POINTER(C.c_uint32)),
                ("records", C.POINTER(C.c_uint32)), ("node_count", C.c_size_t),
                ("emitter_count", C.c_size_t), ("triangle_count", C.c_size_t), ("energy", C.c_double)]


def _p(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


_f, _u, _d = C.c_float, C.c_uint32, C.c_double
lib.or_build_bvh.restype = C.c_size_t
lib.or_compile_meshes.restype = C.c_int
lib.or_bvh_depth.restype = C.c_uint32
lib.or_hash_u32.restype = C.c_uint32
lib.or_hash_combine.restype = C.c_uint32
lib.or_sobol.restype = C.c_uint32
lib.or_sobol_directions.restype = C.POINTER(C.c_uint32)
lib.or_octahedral.restype = C.c_uint32
lib.or_blackbody.restype = C.c_double
lib.or_blackbody.argtypes = [C.c_double, C.c_double]
lib.or_wavelength_pdf.restype = C.c_double
lib.or_wavelength_pdf.argtypes = [C.c_double]
lib.or_sample_wavelengths.argtypes = [C.c_double, C.POINTER(C.c_double)]
lib.or_table_albedo.restype = C.c_double
lib.or_table_albedo.argtypes = [C.c_double, C.c_double, C.c_double]
lib.or_albedo_tables.restype = C.POINTER(C.c_double)
lib.or_pack_lights.restype = C.c_size_t
lib.or_pack_lights_size.restype = C.c_size_t
lib.or_pack_lights_size.argtypes = [C.POINTER(OrLight), C.c_size_t]
lib.or_pack_lights.argtypes = [C.POINTER(OrLight), C.c_size_t, C.c_double, C.POINTER(C.c_float),
                               C.POINTER(C.c_double)]
lib.or_ray_frame.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                             C.c_uint32, C.c_uint32, C.POINTER(OrFrame)]
lib.or_look_frame.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                              C.c_uint32, C.c_uint32, C.c_int, C.POINTER(OrFrame)]


def build_bvh(positions: np.ndarray, indices: np.ndarray):
    """The reference's BVH (bvh.lucb:66-217): nodes, order, and indices in leaf order."""
    positions = np.ascontiguousarray(positions, np.float32)
    indices = np.ascontiguousarray(indices, np.uint32).reshape(-1, 3)
    T = len(indices)
    nodes = np.zeros(2 * max(T, 1), NODE_DTYPE)
    order = np.zeros(max(T, 1), np.uint32)
    n = lib.or_build_bvh(_p(positions, _f), _p(indices, _u), C.c_size_t(T), nodes.ctypes.data_as(C.c_void_p),
                         _p(order, _u))
    return nodes[:n].copy(), order[:T].copy()


def compile_meshes(meshes, library: int) -> dict:
    """compile_scene (scene.lucb:111-129, 253-294, 364-398) with its BVH, over meshes with
    the boundary's fields (positions, indices, faces, face_count, normals,
    normals_per_corner, face_materials, transform; luce_render_b200.MeshData has them):
    the arrays a compiled scene holds -- positions, then indices, shading, faces in leaf
    order, nodes, order."""
    keep = []

    def arr(a, dtype, cols):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype).reshape(-1, cols) if cols else np.ascontiguousarray(a, dtype)
        keep.append(a)
        return a

    descs = (OrMesh * max(1, len(meshes)))()
    points = triangles = 0
    for d, m in zip(descs, meshes):
        pos, tri = arr(m.positions, np.float32, 3), arr(m.indices, np.uint32, 3)
        d.positions, d.point_count = _p(pos, _f), len(pos)
        d.indices, d.triangle_count = _p(tri, _u), len(tri)
        faces = arr(m.faces, np.uint32, 0)
        if faces is not None:
            d.faces = _p(faces, _u)
        d.face_count = int(m.face_count)
        normals = arr(m.normals, np.float32, 3)
        if normals is not None:
            d.normals = _p(normals, _f)
            d.normals_per_corner = 1 if m.normals_per_corner else 0
        mats = arr(m.face_materials, np.uint32, 0)
        if mats is not None:
            d.face_materials = _p(mats, _u)
        if m.transform is not None:
            d.transform[:] = [float(v) for v in np.asarray(m.transform, np.float64).reshape(-1)]
        points += len(pos)
        triangles += len(tri)
    positions = np.zeros((points, 3), np.float32)
    indices = np.zeros((triangles, 3), np.uint32)
    shading = np.zeros((triangles, 4), np.uint32)
    faces = np.zeros(triangles, np.uint32)
    nodes = np.zeros(2 * max(triangles, 1), NODE_DTYPE)
    order = np.zeros(max(triangles, 1), np.uint32)
    count = C.c_size_t()
    status = lib.or_compile_meshes(descs, len(meshes), C.c_size_t(library), _p(positions, _f), _p(indices, _u),
                                   _p(shading, _u), _p(faces, _u), nodes.ctypes.data_as(C.c_void_p), _p(order, _u),
                                   C.byref(count))
    if status != 0:
        raise ValueError("a triangle names a point or polygon its mesh lacks")
    return {"positions": positions, "indices": indices, "shading": shading, "faces": faces,
            "nodes": nodes[: count.value].copy(), "order": order[:triangles].copy()}


def bvh_depth(nodes: np.ndarray) -> int:
    return int(lib.or_bvh_depth(nodes.ctypes.data_as(C.c_void_p), C.c_size_t(len(nodes))))


def trace(nodes, positions, indices, rays, any_hit=False, stack_limit=0, threads=0):
    """The reference's trace_closest / trace_any (bvh.glsl:51-122) over rays (n x 8).
    Returns (hits or booleans, Counts)."""
    rays = np.ascontiguousarray(rays, np.float32)
    positions = np.ascontiguousarray(positions, np.float32)
    indices = np.ascontiguousarray(indices, np.uint32)
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    n = len(rays)
    counts = Counts()
    if any_hit:
        out = np.zeros(n, np.uint8)
        lib.or_trace_any_batch(nodes.ctypes.data_as(C.c_void_p), _p(positions, _f), _p(indices, _u), _p(rays, _f),
                               C.c_size_t(n), stack_limit, _p(out, C.c_uint8), C.byref(counts), threads)
    else:
        out = np.zeros(n, HIT_DTYPE)
        lib.or_trace_closest_batch(nodes.ctypes.data_as(C.c_void_p), _p(positions, _f), _p(indices, _u),
                                   _p(rays, _f), C.c_size_t(n), stack_limit, out.ctypes.data_as(C.c_void_p),
                                   C.byref(counts), threads)
    return out, counts


def nearest_f64(positions, indices, faces, rays, threads=0):
    """tests/gpu/main.lucb:82-119 per ray: (face or -1, distance, margin)."""
    rays = np.ascontiguousarray(rays, np.float32)
    positions = np.ascontiguousarray(positions, np.float32)
    indices = np.ascontiguousarray(indices, np.uint32)
    faces = np.ascontiguousarray(faces, np.uint32)
    n = len(rays)
    face = np.zeros(n, np.int64)
    dist = np.zeros(n, np.float64)
    margin = np.zeros(n, np.float64)
    lib.or_nearest_f64(_p(positions, _f), _p(indices, _u), _p(faces, _u), C.c_size_t(len(indices)), _p(rays, _f),
                       C.c_size_t(n), _p(face, C.c_int64), _p(dist, _d), _p(margin, _d), threads)
    return face, dist, margin


def brute_watertight(positions, indices, ids, rays, any_hit=False, threads=0):
    """FP32 watertight brute force: (prim int32, t, u, v)."""
    rays = np.ascontiguousarray(rays, np.float32)
    positions = np.ascontiguousarray(positions, np.float32)
    indices = np.ascontiguousarray(indices, np.uint32)
    n = len(rays)
    prim = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    u = np.zeros(n, np.float32)
    v = np.zeros(n, np.float32)
    ids_p = None if ids is None else _p(np.ascontiguousarray(ids, np.uint32), _u)
    lib.or_brute_watertight(_p(positions, _f), _p(indices, _u), ids_p, C.c_size_t(len(indices)), _p(rays, _f),
                            C.c_size_t(n), 1 if any_hit else 0, _p(prim, C.c_int32), _p(t, _f), _p(u, _f), _p(v, _f),
                            threads)
    return prim, t, u, v


def probe_rays(block16: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(block16, np.float32)
    w, h = int(b[11]), int(b[15])
    rays = np.zeros((w * h, 8), np.float32)
    lib.or_probe_rays(_p(b, _f), _p(rays, _f))
    return rays


def frame_of_camera(matrix12, projection, focal_length, horizontal_aperture, f_stop, focus_distance, w, h):
    f = OrFrame()
    m = (C.c_double * 12)(*[float(v) for v in matrix12])
    status = lib.or_ray_frame(m, projection, focal_length, horizontal_aperture, f_stop, focus_distance, w, h,
                              C.byref(f))
    return status, f


def look_frame(position, forward, up, tan_half_height, w, h, orthographic=False):
    f = OrFrame()
    p, fw, u = ((C.c_double * 3)(*map(float, v)) for v in (position, forward, up))
    status = lib.or_look_frame(p, fw, u, tan_half_height, w, h, 1 if orthographic else 0, C.byref(f))
    return status, f


def frame_pack(f: OrFrame) -> np.ndarray:
    out = np.zeros(16, np.float32)
    lib.or_frame_pack(C.byref(f), _p(out, _f))
    return out


def frame_ray(f: OrFrame, x, y):
    o = (C.c_double * 3)()
    d = (C.c_double * 3)()
    lib.or_frame_ray(C.byref(f), C.c_double(x), C.c_double(y), o, d)
    return np.array(o[:]), np.array(d[:])


def sobol_directions() -> np.ndarray:
    p = lib.or_sobol_directions()
    return np.array([p[i] for i in range(128)], np.uint32)


def sample4_bits(seed, pixel, index, group) -> np.ndarray:
    out = (C.c_uint32 * 4)()
    lib.or_sample4_bits(C.c_uint32(seed), C.c_uint32(pixel), C.c_uint32(index), C.c_uint32(group), out)
    return np.array(out[:], np.uint32)


def hash_u32(x: int) -> int:
    return int(lib.or_hash_u32(C.c_uint32(x)))


def film_matrix() -> np.ndarray:
    out = (C.c_double * 9)()
    lib.or_film_matrix(out)
    return np.array(out[:]).reshape(3, 3)


def acescg_to_xyz_e() -> np.ndarray:
    out = (C.c_double * 9)()
    lib.or_acescg_to_xyz_e(out)
    return np.array(out[:]).reshape(3, 3)


def cmf(lam: float) -> np.ndarray:
    out = (C.c_double * 3)()
    lib.or_cmf(C.c_double(lam), out)
    return np.array(out[:])


def cmf_integrals() -> np.ndarray:
    out = (C.c_double * 3)()
    lib.or_cmf_integrals(out)
    return np.array(out[:])


def fit_spectrum(rgb) -> np.ndarray:
    out = (C.c_double * 4)()
    lib.or_fit_spectrum((C.c_double * 3)(*map(float, rgb)), out)
    return np.array(out[:])


def blackbody_xyz(kelvin: float) -> np.ndarray:
    out = (C.c_double * 3)()
    lib.or_blackbody_xyz(C.c_double(kelvin), out)
    return np.array(out[:])


def sample_wavelengths(u: float) -> np.ndarray:
    out = (C.c_double * 4)()
    lib.or_sample_wavelengths(u, out)
    return np.array(out[:])


def wavelength_pdf(lam: float) -> float:
    return float(lib.or_wavelength_pdf(lam))


def octahedral(n) -> int:
    return int(lib.or_octahedral((C.c_double * 3)(*map(float, n))))


def octahedral_decode(packed: int) -> np.ndarray:
    out = (C.c_double * 3)()
    lib.or_octahedral_decode(C.c_uint32(packed), out)
    return np.array(out[:])


ALBEDO_TABLE_SIZE = 32 * 32 + 32 + 32 * 32 * 16


def table_albedo(mu: float, roughness: float, eta: float) -> float:
    """One node of the albedo tables (tables.comp:21-36): the mean of F G2 / G1 over a
    32 x 32 grid of visible normals at view cosine mu; eta <= 0 for F = 1."""
    return lib.or_table_albedo(mu, roughness, eta)


def albedo_tables() -> np.ndarray:
    """The whole table (E_ggx 32 x 32, its average over mu, E_dielectric 16 x 32 x 32),
    laid out as the kernels read it (microfacet.glsl:67-74)."""
    ptr = lib.or_albedo_tables()
    return np.ctypeslib.as_array(ptr, shape=(ALBEDO_TABLE_SIZE,)).copy()


def material_standard() -> OrMaterial:
    m = OrMaterial()
    lib.or_material_standard(C.byref(m))
    return m


def material_from(openpbr) -> OrMaterial:
    """An oracle material with the same fields as a luce_render_b200.OpenPbr."""
    m = OrMaterial()
    for name, _ in OrMaterial._fields_:
        value = getattr(openpbr, name)
        if hasattr(value, "__len__"):
            getattr(m, name)[:] = list(value)
        else:
            setattr(m, name, value)
    return m


def pack_material(m: OrMaterial, program: float = -1.0) -> np.ndarray:
    out = np.zeros(64, np.float32)
    lib.or_pack_material(C.byref(m), C.c_float(program), _p(out, _f))
    return out


def light_from(l) -> OrLight:
    o = OrLight()
    for name, _ in OrLight._fields_:
        value = getattr(l, name)
        if hasattr(value, "__len__"):
            getattr(o, name)[:] = list(value)
        else:
            setattr(o, name, value)
    return o


def pack_lights(lights, radius: float, with_image: bool = False):
    """pack_lights (lights.lucb:29-131): (records n x 28, distant and dome power); with
    `with_image`, the flat rows with the textured dome's texels and cumulative weights
    after the records, and the light count: (rows, power, n)."""
    arr = (OrLight * max(1, len(lights)))(*[light_from(l) for l in lights])
    out = np.zeros(max(28, lib.or_pack_lights_size(arr, len(lights))), np.float32)
    power = C.c_double()
    n = lib.or_pack_lights(arr, len(lights), radius, _p(out, _f), C.byref(power))
    if with_image:
        return out, power.value, n
    return out[: n * 28].reshape(-1, 28).copy(), power.value


def light_tree(positions, indices, shading, light_rows, materials):
    """build_light_tree (light_tree.lucb:91-199): dict of nodes, links, records, counts."""
    positions = np.ascontiguousarray(positions, np.float32)
    indices = np.ascontiguousarray(indices, np.uint32)
    shading = np.ascontiguousarray(shading, np.uint32)
    rows = np.ascontiguousarray(light_rows, np.float32).reshape(-1)
    lib_mats = (OrMaterial * max(1, len(materials)))(*materials)
    tree = OrTree()
    T = len(indices) // 3 if indices.ndim == 1 else len(indices)
    lib.or_build_light_tree(_p(positions, _f), _p(indices, _u), _p(shading, _u), C.c_size_t(T), _p(rows, _f),
                            C.c_size_t(len(rows) // 28), lib_mats, C.c_size_t(len(materials)), C.byref(tree))
    n, e = tree.node_count, tree.emitter_count
    out = {
        "nodes": np.array([tree.nodes[i] for i in range(n * 12)], np.float32).reshape(-1, 12),
        "links": np.array([tree.links[i] for i in range(n * 2)], np.uint32).reshape(-1, 2),
        "records": np.array([tree.records[i] for i in range(e * 4 + T)], np.uint32),
        "emitter_count": int(e),
        "node_count": int(n),
        "energy": float(tree.energy),
    }
    lib.or_light_tree_free(C.byref(tree))
    return out


class RenderDesc(C.Structure):
    _fields_ = [("positions", C.POINTER(C.c_float)), ("indices", C.POINTER(C.c_uint32)),
                ("shading", C.POINTER(C.c_uint32)), ("triangle_count", C.c_size_t), ("nodes", C.c_void_p),
                ("light_rows", C.POINTER(C.c_float)), ("light_count", C.c_uint32),
                ("tree_nodes", C.POINTER(C.c_float)), ("tree_links", C.POINTER(C.c_uint32)),
                ("tree_records", C.POINTER(C.c_uint32)), ("tree_node_count", C.c_uint32),
                ("emitter_count", C.c_uint32), ("materials", C.POINTER(C.c_float)), ("p_distant", C.c_double),
                ("background_fit", C.c_float * 4), ("background_rgb", C.c_float * 3), ("film", C.c_double * 9),
                ("cmf_integrals", C.c_double * 3), ("frame", C.c_float * 16), ("lens_radius", C.c_double),
                ("focus_distance", C.c_double), ("forward", C.c_double * 3), ("width", C.c_uint32),
                ("height", C.c_uint32), ("max_bounces", C.c_uint32), ("spectral", C.c_uint32), ("seed", C.c_uint32),
                ("limits", C.c_double * 3), ("clamp", C.c_double), ("light_paths", C.c_uint32),
                ("light_band", C.c_uint32), ("pixel_area_inv", C.c_double), ("emit_share", C.c_double),
                ("emit_radius", C.c_double), ("emit_center", C.c_double * 3), ("through", C.c_uint32)]


def render(arrays: dict, lights, library, frame, samples: int, max_bounces: int, spectral: bool, seed: int = 1,
           background=(0.0, 0.0, 0.0), clamp: float = 0.0, limits=(1024.0, 1024.0, 1024.0), threads: int = 0,
           light_tracing: float = 0.0, pool: int = 0):
    """The f64 estimator over a compiled scene's arrays (leaf order), the scene's lights
    (luce_render_b200.Light), the material library (default first, OrMaterial or
    luce_render_b200.OpenPbr) and a luce_render_b200.Frame. Returns (mean, variance),
    each height x width x 3 (ACEScg); with light tracing, of each sample's image (camera
    values plus that sample's light paths' splats)."""
    job = RenderJob(arrays, lights, library, frame, max_bounces, spectral, seed, background, clamp, limits,
                    light_tracing, pool)
    n = frame.width * frame.height
    if job.light_paths:
        mean, var, _ = job.traced(samples, 0, threads)
    else:
        mean, var, _ = job.region(samples, 0, 0, n, threads)
    return mean.reshape(frame.height, frame.width, 3), var.reshape(frame.height, frame.width, 3)


def light_paths(light_tracing: float, pixels: int, pool: int, orthographic: bool, emitters: int, afar: bool = False):
    """Loaded.light_paths (loading.lucb:163-168) and the band they follow: light tracing's
    share of the pixels (at least one), at most a band's; none for an orthographic camera
    or a scene with neither emitters nor light paths from afar. Returns (light paths,
    band)."""
    band = min(pool if pool > 0 else 2097152, pixels)
    if light_tracing <= 0.0 or orthographic or (emitters == 0 and not afar):
        return 0, band
    wanted = max(1, int(math.floor(light_tracing * pixels + 0.5)))
    return min(wanted, band), band


class RenderJob:
    """A prepared f64 render: the loaded records built once, then any pixel range."""

    def __init__(self, arrays: dict, lights, library, frame, max_bounces: int, spectral: bool, seed: int = 1,
                 background=(0.0, 0.0, 0.0), clamp: float = 0.0, limits=(1024.0, 1024.0, 1024.0),
                 light_tracing: float = 0.0, pool: int = 0):
        self.desc, self.keep = _render_desc(arrays, lights, library, frame, max_bounces, spectral, seed, background,
                                            clamp, limits, light_tracing)
        count, band = light_paths(light_tracing, frame.width * frame.height, pool, bool(frame.orthographic),
                                  self.desc.emitter_count, self.desc.emit_share > 0.0)
        self.light_paths = count
        self.desc.light_paths, self.desc.light_band = count, band
        area = float(np.linalg.norm(np.array(frame.du)) * np.linalg.norm(np.array(frame.dv)))
        self.desc.pixel_area_inv = 1.0 / area if area > 0.0 else 0.0
        self.pixels = frame.width * frame.height

    def traced(self, samples: int, sample_first: int = 0, threads: int = 0):
        """All pixels with light tracing, samples [sample_first, + samples): (mean, var,
        (closest rays, shadow rays)) of the per-sample images."""
        mean = np.zeros(self.pixels * 3, np.float64)
        var = np.zeros(self.pixels * 3, np.float64)
        rays = (C.c_uint64 * 2)()
        lib.or_render_traced(C.byref(self.desc), C.c_uint32(samples), C.c_uint32(sample_first), _p(mean, C.c_double),
                             _p(var, C.c_double), rays, threads)
        return mean.reshape(-1, 3), var.reshape(-1, 3), (int(rays[0]), int(rays[1]))

    def region(self, samples: int, sample_first: int, first: int, count: int, threads: int = 0):
        """Pixels [first, first + count), samples [sample_first, + samples): (mean, var,
        (closest rays, shadow rays))."""
        mean = np.zeros(count * 3, np.float64)
        var = np.zeros(count * 3, np.float64)
        rays = (C.c_uint64 * 2)()
        lib.or_render_region(C.byref(self.desc), C.c_uint32(samples), C.c_uint32(sample_first), C.c_size_t(first),
                             C.c_size_t(count), _p(mean, C.c_double), _p(var, C.c_double), rays, threads)
        return mean.reshape(-1, 3), var.reshape(-1, 3), (int(rays[0]), int(rays[1]))


def casts_caustics(m) -> bool:
    """casts_caustics (loading.lucb:215-219): it refracts, or reflects sharply enough."""
    if m.transmission_weight > 0.0:
        return True
    if m.base_metalness > 0.0 and m.specular_roughness < 0.3:
        return True
    if m.coat_weight > 0.0 and m.coat_roughness < 0.3:
        return True
    return m.specular_weight > 0.0 and m.specular_roughness < 0.1


def caster_bounds(positions, indices, shading, materials):
    """caster_bounds (loading.lucb:224-241): (centre, radius) of the triangles whose
    material casts caustics, or None."""
    cast = np.array([casts_caustics(m) for m in materials], bool)
    mat = np.asarray(shading, np.uint32).reshape(-1, 4)[:, 3]
    chosen = (mat < len(materials)) & cast[np.minimum(mat, len(materials) - 1)]
    if not chosen.any():
        return None
    corners = np.asarray(indices, np.uint32).reshape(-1, 3)[chosen].reshape(-1)
    pts = np.asarray(positions, np.float32).reshape(-1, 3)[corners].astype(np.float64)
    lo, hi = pts.min(0), pts.max(0)
    return (lo + hi) * 0.5, max(1e-3, 0.5 * float(np.linalg.norm(hi - lo)))


def _render_desc(arrays, lights, library, frame, max_bounces, spectral, seed, background, clamp, limits,
                 light_tracing=0.0):
    positions = np.ascontiguousarray(arrays["positions"], np.float32).reshape(-1)
    indices = np.ascontiguousarray(arrays["indices"], np.uint32).reshape(-1)
    shading = np.ascontiguousarray(arrays["shading"], np.uint32).reshape(-1)
    nodes = np.ascontiguousarray(arrays["nodes"], NODE_DTYPE)
    T = len(indices) // 3
    root = nodes[0]
    radius = 1.0
    if T and root["lo"][0] <= root["hi"][0]:
        d = (root["hi"].astype(np.float64) - root["lo"].astype(np.float64))
        radius = max(1.0, 0.5 * float(np.sqrt((d * d).sum())))
    flat_rows, distant_power, light_count = pack_lights(list(lights), radius, with_image=True)
    rows = flat_rows[: light_count * 28].reshape(-1, 28)
    mats = [m if isinstance(m, OrMaterial) else material_from(m) for m in library]
    tree = light_tree(positions, indices, shading, rows, mats)
    total = distant_power + tree["energy"]
    if tree["emitter_count"] > 0:
        p_distant = distant_power / total if total > 0 else 0.0
    else:
        p_distant = 1.0 if distant_power > 0 else 0.0
    material_rows = np.concatenate([pack_material(m) for m in mats]).astype(np.float32)
    rows = np.ascontiguousarray(flat_rows, np.float32)
    tnodes = np.ascontiguousarray(tree["nodes"].reshape(-1), np.float32)
    tlinks = np.ascontiguousarray(tree["links"].reshape(-1), np.uint32)
    trec = np.ascontiguousarray(tree["records"], np.uint32)
    keep = [positions, indices, shading, nodes, rows, tnodes, tlinks, trec, material_rows]
    r = RenderDesc()
    r.positions, r.indices, r.shading = _p(positions, _f), _p(indices, _u), _p(shading, _u)
    r.triangle_count = T
    r.nodes = nodes.ctypes.data_as(C.c_void_p)
    r.light_rows = _p(rows, _f)
    r.light_count = light_count
    r.tree_nodes = _p(tnodes, _f) if len(tnodes) else None
    r.tree_links = _p(tlinks, _u) if len(tlinks) else None
    r.tree_records = _p(trec, _u) if len(trec) else None
    r.tree_node_count = tree["node_count"]
    r.emitter_count = tree["emitter_count"]
    r.materials = _p(material_rows, _f)
    r.p_distant = p_distant
    r.background_fit[:] = [float(x) for x in fit_spectrum(background)]
    r.background_rgb[:] = [float(x) for x in background]
    r.film[:] = list(film_matrix().reshape(-1))
    r.cmf_integrals[:] = list(cmf_integrals())
    r.frame[:] = [float(x) for x in frame.pack()]
    r.lens_radius = frame.lens_radius
    r.focus_distance = frame.focus_distance
    r.forward[:] = list(frame.forward)
    r.width, r.height = frame.width, frame.height
    r.max_bounces = max_bounces
    r.spectral = 1 if spectral else 0
    r.seed = seed
    r.limits[:] = [float(x) for x in limits]
    # Cut-outs (loading.lucb:121-124, 161): 8 rounds more when a material the triangles
    # use has geometry_opacity below 1.
    used = set(int(x) for x in np.asarray(shading, np.uint32).reshape(-1, 4)[:, 3]) if T else set()
    r.through = 8 if any(i < len(mats) and mats[i].geometry_opacity < 1.0 for i in used) else 0
    # Light paths from afar (loading.lucb:127-146): domes and distant lights with a size
    # share light paths with the tree's emitters by power, on a disk around what casts
    # caustics.
    sized = any(row[3] == 4.0 or (row[3] == 3.0 and row[11] < np.float32(1.0) - np.float32(1e-7))
                for row in flat_rows[: light_count * 28].reshape(-1, 28))
    r.emit_share, r.emit_radius = 0.0, 1.0
    if sized and light_tracing > 0.0 and not frame.orthographic:
        found = caster_bounds(positions, indices, shading, mats)
        if found is not None:
            center, reach = found
            afar_power = distant_power * (reach / radius) ** 2
            both = afar_power + tree["energy"]
            r.emit_share = afar_power / both if both > 0.0 else 0.0
            r.emit_radius = reach
            r.emit_center[:] = [float(x) for x in center]
    r.clamp = clamp
    return r, keep
