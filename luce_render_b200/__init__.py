"""luce_render_b200: a B200-native (sm_100a) implementation of luce-render's wavefront
path-tracing hot path, behind a C ABI (include/luce_render_b200.h).

This module is the ctypes harness over that ABI, mirroring luce-render's ``render``
package for the path (package.prisma:13):

=====================================  ===============================================
luce-render (src/render/...)            here
=====================================  ===============================================
``compile_scene`` (scene.lucb:111)      :func:`compile_scene` -> :class:`CompiledScene`
``GpuScene.upload`` (device.lucb:41)    :meth:`GpuScene.upload`
``probe`` (device.lucb:138)             :func:`probe`
``ray_frame`` / ``look_frame``          :func:`ray_frame` / :func:`look_frame`
(camera.lucb:57, 84)
``RenderSettings.of`` (integr.:84)      :meth:`RenderSettings.of`
``Renderer.create/advance/finish/       :class:`Renderer`
samples_done/image/read``
=====================================  ===============================================

Errors raise :class:`RenderError` with the reference's codes (400 invalid, 401 limit,
402 stopped; module.lucb:60-63) or 500/504 for device failures. The CUDA library is
required: importing this package fails loudly when it has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Iterable, Sequence

import numpy as np

_HERE = Path(__file__).resolve().parent
LIBRARY_PATH = _HERE / "libluce_render_b200.so"

INVALID, LIMIT, STOPPED, DEVICE, TIMEOUT = 400, 401, 402, 500, 504
TRACE_ANY, TRACE_REFERENCE, TRACE_COUNT = 1, 2, 4
LIGHT_RECT, LIGHT_DISK, LIGHT_SPHERE, LIGHT_DISTANT, LIGHT_DOME = 0, 1, 2, 3, 4
REFIT_DEVICE = 1
COMPILE_NO_TREES = 1


class RenderError(RuntimeError):
    """A failing call of the C ABI: ``code`` is its status, the message its text."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


def _missing() -> str:
    return (f"{LIBRARY_PATH} is missing: build it with `python luce_render_b200/build.py` "
            "(nvcc for sm_100a). There is no CPU fallback.")


if not LIBRARY_PATH.exists():
    raise ImportError(_missing())


class _Library:
    """The C-ABI library, mapped into the process at the first call through it.

    Describing a workload -- MeshData, camera(), light(), OpenPbr and the scene
    generators of :mod:`luce_render_b200.scenes` -- calls nothing in it, so a process
    that only builds inputs (the benchmark's CPU reference arm) never maps it. Every
    compile, upload, trace and render goes through it; there is no CPU fallback: the
    package refuses to import without the library, and a library that fails to load
    raises at that first call."""

    def __init__(self):
        self._dll = None

    def _open(self) -> C.CDLL:
        if self._dll is None:
            if not LIBRARY_PATH.exists():
                raise ImportError(_missing())
            dll = C.CDLL(str(LIBRARY_PATH))
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(dll, name, None)
                if fn is not None:
                    fn.restype = res
                    fn.argtypes = args
            self._dll = dll
        return self._dll

    def __getattr__(self, name: str):
        if name.startswith("__"):
            raise AttributeError(name)
        fn = getattr(self._open(), name)
        setattr(self, name, fn)  # later calls skip this lookup
        return fn


lib = _Library()


# ---- structures (include/luce_render_b200.h) ------------------------------------------

class Mesh(C.Structure):
    _fields_ = [("positions", C.POINTER(C.c_float)), ("point_count", C.c_uint64),
                ("indices", C.POINTER(C.c_uint32)), ("triangle_count", C.c_uint64),
                ("triangle_faces", C.POINTER(C.c_uint32)), ("face_count", C.c_uint32),
                ("normals", C.POINTER(C.c_float)), ("normals_per_corner", C.c_int32),
                ("face_materials", C.POINTER(C.c_uint32)), ("transform", C.c_double * 12)]


class Camera(C.Structure):
    _fields_ = [("matrix", C.c_double * 12), ("projection", C.c_int32), ("focal_length", C.c_double),
                ("horizontal_aperture", C.c_double), ("f_stop", C.c_double), ("focus_distance", C.c_double)]


class Light(C.Structure):
    _fields_ = [("matrix", C.c_double * 12), ("shape", C.c_int32), ("color", C.c_double * 3),
                ("intensity", C.c_double), ("exposure", C.c_double), ("temperature", C.c_double),
                ("width", C.c_double), ("height", C.c_double), ("radius", C.c_double), ("angle", C.c_double),
                ("normalize", C.c_int32), ("visible", C.c_int32), ("image", C.POINTER(C.c_float)),
                ("image_width", C.c_uint32), ("image_height", C.c_uint32)]


class OpenPbr(C.Structure):
    _fields_ = [("base_weight", C.c_double), ("base_color", C.c_double * 3), ("base_metalness", C.c_double),
                ("base_diffuse_roughness", C.c_double), ("specular_weight", C.c_double),
                ("specular_color", C.c_double * 3), ("specular_roughness", C.c_double),
                ("specular_roughness_anisotropy", C.c_double), ("specular_ior", C.c_double),
                ("transmission_weight", C.c_double), ("transmission_color", C.c_double * 3),
                ("coat_weight", C.c_double), ("coat_color", C.c_double * 3), ("coat_roughness", C.c_double),
                ("coat_roughness_anisotropy", C.c_double), ("coat_ior", C.c_double),
                ("coat_darkening", C.c_double), ("emission_luminance", C.c_double),
                ("emission_color", C.c_double * 3), ("geometry_opacity", C.c_double),
                ("geometry_thin_walled", C.c_int32), ("transmission_dispersion_scale", C.c_double),
                ("transmission_dispersion_abbe_number", C.c_double)]

    @staticmethod
    def standard() -> "OpenPbr":
        """OpenPbr.standard (materials.lucb:46-53): the values lr_openpbr_standard sets,
        filled here so that describing a material maps no library (a CPU test holds the
        two equal)."""
        m = OpenPbr()
        m.base_weight = 1.0
        m.base_color[:] = [0.8, 0.8, 0.8]
        for name in ("specular_color", "transmission_color", "coat_color", "emission_color"):
            getattr(m, name)[:] = [1.0, 1.0, 1.0]
        m.specular_weight, m.specular_roughness, m.specular_ior = 1.0, 0.3, 1.5
        m.coat_ior, m.coat_darkening = 1.6, 1.0
        m.geometry_opacity = 1.0
        m.transmission_dispersion_abbe_number = 20.0
        return m

    @staticmethod
    def lambert(color=(0.8, 0.8, 0.8), emission: float = 0.0, emission_color=(1.0, 1.0, 1.0),
                roughness: float = 0.0) -> "OpenPbr":
        """A diffuse-only material: the standard one with specular_weight 0."""
        m = OpenPbr.standard()
        m.base_color[:] = list(color)
        m.specular_weight = 0.0
        m.base_diffuse_roughness = roughness
        m.emission_luminance = emission
        m.emission_color[:] = list(emission_color)
        return m


class BvhNode(C.Structure):
    _fields_ = [("lo", C.c_float * 3), ("first", C.c_uint32), ("hi", C.c_float * 3), ("count", C.c_uint32)]


NODE_DTYPE = np.dtype([("lo", "<f4", 3), ("first", "<u4"), ("hi", "<f4", 3), ("count", "<u4")])


class SceneInfo(C.Structure):
    _fields_ = [("point_count", C.c_uint64), ("triangle_count", C.c_uint64), ("node_count", C.c_uint64),
                ("face_count", C.c_uint32), ("camera_count", C.c_uint32), ("light_count", C.c_uint32),
                ("material_count", C.c_uint32), ("bvh_depth", C.c_uint32)]


class GpuSceneInfo(C.Structure):
    _fields_ = [("bytes", C.c_uint64), ("bvh2_depth", C.c_uint32), ("wide4_nodes", C.c_uint64),
                ("wide8_nodes", C.c_uint64), ("wide4_stack", C.c_uint32), ("wide8_stack", C.c_uint32),
                ("width", C.c_uint32), ("stack", C.c_uint32)]


class Frame(C.Structure):
    """RayFrame (camera.lucb:26-54)."""
    _fields_ = [("position", C.c_double * 3), ("corner", C.c_double * 3), ("du", C.c_double * 3),
                ("dv", C.c_double * 3), ("forward", C.c_double * 3), ("orthographic", C.c_int32),
                ("width", C.c_uint32), ("height", C.c_uint32), ("lens_radius", C.c_double),
                ("focus_distance", C.c_double)]

    def pack(self) -> np.ndarray:
        """RayFrame.pack (camera.lucb:41-47): the 16 floats the kernels read."""
        out = np.zeros(16, np.float32)
        _check(lib.lr_frame_pack(C.byref(self), _fptr(out)))
        return out

    def ray(self, x: float, y: float):
        """RayFrame.ray (camera.lucb:51-54): origin and unnormalized direction, f64."""
        film = np.array(self.corner) + np.array(self.du) * x + np.array(self.dv) * y
        if self.orthographic:
            return np.array(self.position) + film, np.array(self.forward)
        return np.array(self.position), film


class Settings(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("samples", C.c_uint32),
                ("max_bounces", C.c_uint32), ("spectral", C.c_int32), ("camera", C.c_int32),
                ("background", C.c_double * 3), ("material", OpenPbr), ("pool", C.c_uint32),
                ("seed", C.c_uint32), ("software_bvh", C.c_int32), ("diffuse_bounces", C.c_uint32),
                ("glossy_bounces", C.c_uint32), ("transmission_bounces", C.c_uint32),
                ("clamp_indirect", C.c_double), ("noise_threshold", C.c_double),
                ("adaptive_minimum", C.c_uint32), ("profile", C.c_int32), ("guiding", C.c_int32),
                ("light_tracing", C.c_double)]


class RenderStats(C.Structure):
    _fields_ = [("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("shaded", C.c_uint64),
                ("passes", C.c_uint64), ("closest_nodes", C.c_uint64), ("closest_tests", C.c_uint64),
                ("shadow_nodes", C.c_uint64), ("shadow_tests", C.c_uint64)]


# ---- signatures ---------------------------------------------------------------------------

class BatchSettings(C.Structure):
    """lr_batch_settings: paths a pass, the most bounces a member may ask for, the most
    members at once, profiling."""
    _fields_ = [("pool", C.c_uint32), ("max_bounces", C.c_uint32), ("capacity", C.c_uint32),
                ("profile", C.c_int32)]

    @staticmethod
    def default(**overrides) -> "BatchSettings":
        b = BatchSettings()
        lib.lr_batch_settings_default(C.byref(b))
        for key, value in overrides.items():
            setattr(b, key, value)
        return b


class BatchTuning(C.Structure):
    """lr_batch_tuning: the BVH width and paths a pass the autotuner chose, the chosen
    candidate's measured rate and how many candidates it timed."""
    _fields_ = [("width", C.c_uint32), ("fill", C.c_uint32), ("paths_per_ms", C.c_double),
                ("candidates", C.c_uint32), ("class_width", C.c_uint32 * 3), ("class_members", C.c_uint32 * 3),
                ("class_stack", C.c_uint32 * 3), ("class_block", C.c_uint32 * 3), ("bin_interval", C.c_uint32),
                ("refill_at", C.c_uint32), ("thin_from", C.c_int32)]


class ServerSettings(C.Structure):
    """lr_server_settings."""
    _fields_ = [("device", C.c_int32), ("budget_bytes", C.c_uint64), ("capacity", C.c_uint32),
                ("pool", C.c_uint32), ("max_bounces", C.c_uint32), ("probe_priority", C.c_int32)]

    @staticmethod
    def default(**overrides) -> "ServerSettings":
        s = ServerSettings()
        lib.lr_server_settings_default(C.byref(s))
        for key, value in overrides.items():
            setattr(s, key, value)
        return s


class RequestInfo(C.Structure):
    """lr_request_info."""
    _fields_ = [("kind", C.c_int32), ("state", C.c_int32), ("status", C.c_int32), ("scene", C.c_uint32),
                ("pixels", C.c_uint64), ("samples", C.c_uint32), ("samples_done", C.c_uint32),
                ("submitted", C.c_double), ("admitted", C.c_double), ("first", C.c_double),
                ("finished", C.c_double)]


class ServerStats(C.Structure):
    """lr_server_stats."""
    _fields_ = [(n, C.c_uint64) for n in ("sessions_done", "probes_done", "failed", "pixel_samples", "probe_rays",
                                          "uploads", "evictions", "queued", "live", "scenes_resident",
                                          "bytes_in_use")] + [("seconds", C.c_double), ("tunings", C.c_uint64),
                                                              ("passes", C.c_uint64)] + [
        (n, C.c_double) for n in ("seconds_advance", "seconds_wait", "seconds_progress", "seconds_admit", "seconds_tune")]


_vp, _i32, _u32, _u64, _sz = C.c_void_p, C.c_int32, C.c_uint32, C.c_uint64, C.c_size_t
_SIGNATURES = {
    "lr_last_error": (C.c_char_p, []),
    "lr_version": (C.c_char_p, []),
    "lr_context_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "lr_context_destroy": (None, [_vp]),
    "lr_context_synchronize": (C.c_int, [_vp]),
    "lr_context_stream": (_vp, [_vp]),
    "lr_device_alloc": (C.c_int, [_vp, _sz, C.POINTER(_vp)]),
    "lr_device_free": (C.c_int, [_vp, _vp]),
    "lr_memcpy_htod": (C.c_int, [_vp, _vp, _vp, _sz]),
    "lr_memcpy_dtoh": (C.c_int, [_vp, _vp, _vp, _sz]),
    "lr_memset_device": (C.c_int, [_vp, _vp, C.c_int, _sz]),
    "lr_host_alloc_pinned": (C.c_int, [_sz, C.POINTER(_vp)]),
    "lr_host_free_pinned": (C.c_int, [_vp]),
    "lr_timer_start": (C.c_int, [_vp]),
    "lr_timer_stop": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "lr_openpbr_standard": (None, [C.POINTER(OpenPbr)]),
    "lr_scene_compile": (C.c_int, [C.POINTER(Mesh), _sz, C.POINTER(Camera), _sz, C.POINTER(Light), _sz,
                                   C.POINTER(OpenPbr), _sz, C.POINTER(_vp)]),
    "lr_scene_compile_ex": (C.c_int, [C.POINTER(Mesh), _sz, C.POINTER(Camera), _sz, C.POINTER(Light), _sz,
                                      C.POINTER(OpenPbr), _sz, _u32, C.POINTER(_vp)]),
    "lr_scene_free": (None, [_vp]),
    "lr_scene_info_get": (C.c_int, [_vp, C.POINTER(SceneInfo)]),
    "lr_scene_arrays": (C.c_int, [_vp] + [C.POINTER(_vp)] * 6),
    "lr_ray_frame": (C.c_int, [C.POINTER(Camera), _u32, _u32, C.POINTER(Frame)]),
    "lr_look_frame": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                C.c_double, _u32, _u32, _i32, C.POINTER(Frame)]),
    "lr_frame_pack": (C.c_int, [C.POINTER(Frame), C.POINTER(C.c_float)]),
    "lr_scene_camera": (C.c_int, [_vp, _i32, C.POINTER(Camera)]),
    "lr_gpu_scene_upload": (C.c_int, [_vp, _vp, C.POINTER(_vp)]),
    "lr_gpu_scene_build": (C.c_int, [_vp, _vp, C.POINTER(_vp)]),
    "lr_gpu_scene_destroy": (None, [_vp]),
    "lr_scene_move_points": (C.c_int, [_vp, C.POINTER(C.c_float), _u64]),
    "lr_gpu_scene_refit": (C.c_int, [_vp, _vp, _vp, _u64, _u32]),
    "lr_renderer_refit": (C.c_int, [_vp, _vp, C.POINTER(Frame)]),
    "lr_gpu_scene_info_get": (C.c_int, [_vp, C.POINTER(GpuSceneInfo)]),
    "lr_probe": (C.c_int, [_vp, _vp, C.POINTER(Frame), _u32, C.POINTER(C.c_uint32), C.POINTER(C.c_float)]),
    "lr_probe_static": (C.c_int, [_vp, _vp, C.POINTER(Frame), _u32, C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_float)]),
    "lr_trace_rays": (C.c_int, [_vp, _vp, C.POINTER(C.c_float), _u64, C.POINTER(C.c_float), _u32]),
    "lr_trace_rays_device": (C.c_int, [_vp, _vp, _vp, _u64, _vp, _u32]),
    "lr_trace_counts": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "lr_settings_default": (None, [C.POINTER(Settings), _u32, _u32, _u32]),
    "lr_renderer_create": (C.c_int, [_vp, _vp, C.POINTER(Settings), C.POINTER(_vp)]),
    "lr_renderer_create_viewed": (C.c_int, [_vp, _vp, C.POINTER(Settings), C.POINTER(Frame), C.POINTER(_vp)]),
    "lr_renderer_advance": (C.c_int, [_vp, C.POINTER(_i32)]),
    "lr_renderer_finish": (C.c_int, [_vp]),
    "lr_renderer_samples_done": (_u32, [_vp]),
    "lr_renderer_passes": (C.c_int, [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    "lr_renderer_image": (C.c_int, [_vp, C.POINTER(_vp)]),
    "lr_renderer_read": (C.c_int, [_vp, C.POINTER(C.c_float), _u64]),
    "lr_renderer_set_samples": (C.c_int, [_vp, _u32]),
    "lr_renderer_join": (C.c_int, [_vp]),
    "lr_renderer_read_async": (C.c_int, [_vp, C.POINTER(C.c_float), _u64]),
    "lr_renderer_restart": (C.c_int, [_vp, C.POINTER(Frame)]),
    "lr_renderer_reload": (C.c_int, [_vp, _vp, C.POINTER(Settings), C.POINTER(Frame)]),
    "lr_renderer_replace_scene": (C.c_int, [_vp, _vp, C.POINTER(Settings), C.POINTER(Frame)]),
    "lr_renderer_display": (C.c_int, [_vp, C.POINTER(_vp)]),
    "lr_renderer_shown_size": (C.c_int, [_vp, C.POINTER(C.c_uint32)]),
    "lr_renderer_set_display": (C.c_int, [_vp, C.c_double, C.c_int]),
    "lr_renderer_converged_pixels": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "lr_renderer_read_wait": (C.c_int, [_vp]),
    "lr_renderer_read_ticket": (C.c_int, [_vp, C.POINTER(C.c_float), _u64, C.POINTER(C.c_uint64)]),
    "lr_renderer_read_landed": (C.c_int, [_vp, _u64, C.POINTER(C.c_int32)]),
    "lr_batch_read_async": (C.c_int, [_vp, _u32, C.POINTER(C.c_float), _u64]),
    "lr_batch_read_wait": (C.c_int, [_vp]),
    "lr_batch_read_ticket": (C.c_int, [_vp, _u32, C.POINTER(C.c_float), _u64, C.POINTER(C.c_uint64)]),
    "lr_batch_read_landed": (C.c_int, [_vp, _u64, C.POINTER(C.c_int32)]),
    "lr_batch_join": (C.c_int, [_vp]),
    "lr_renderer_kernel_times": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "lr_renderer_stats": (C.c_int, [_vp, C.POINTER(RenderStats)]),
    "lr_context_memory": (C.c_int, [_vp, C.c_int32, C.POINTER(C.c_uint64)]),
    "lr_launch_overhead": (C.c_int, [_vp, _u32, C.c_int32, C.POINTER(C.c_double)]),
    "lr_renderer_recorded_rays": (C.c_int, [_vp, _u32, C.c_int32, C.POINTER(C.c_float), _u64,
                                            C.POINTER(C.c_uint64)]),
    "lr_renderer_destroy": (None, [_vp]),
    "lr_albedo_tables": (C.c_int, [_vp, C.POINTER(C.c_float), _sz]),
    "lr_batch_settings_default": (None, [C.POINTER(BatchSettings)]),
    "lr_batch_create": (C.c_int, [_vp, C.POINTER(BatchSettings), C.POINTER(_vp)]),
    "lr_batch_add": (C.c_int, [_vp, _vp, _vp, C.POINTER(Settings), C.POINTER(Frame), C.POINTER(C.c_uint32)]),
    "lr_batch_remove": (C.c_int, [_vp, _u32]),
    "lr_batch_advance": (C.c_int, [_vp, C.POINTER(_i32)]),
    "lr_batch_finish": (C.c_int, [_vp]),
    "lr_batch_member_info": (C.c_int, [_vp, _u32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                       C.POINTER(C.c_uint32)]),
    "lr_batch_set_samples": (C.c_int, [_vp, _u32, _u32]),
    "lr_batch_image": (C.c_int, [_vp, _u32, C.POINTER(_vp)]),
    "lr_batch_read": (C.c_int, [_vp, _u32, C.POINTER(C.c_float), _u64]),
    "lr_batch_tune": (C.c_int, [_vp, C.POINTER(BatchTuning)]),
    "lr_batch_passes": (C.c_int, [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "lr_batch_kernel_times": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "lr_batch_stats": (C.c_int, [_vp, C.POINTER(RenderStats)]),
    "lr_batch_destroy": (None, [_vp]),
    "lr_context_create_ex": (C.c_int, [C.c_int, C.c_int, C.POINTER(_vp)]),
    "lr_batch_wait": (C.c_int, [_vp, C.POINTER(_i32)]),
    "lr_server_settings_default": (None, [C.POINTER(ServerSettings)]),
    "lr_server_create": (C.c_int, [C.POINTER(ServerSettings), C.POINTER(_vp)]),
    "lr_server_add_scene": (C.c_int, [_vp, _vp, C.POINTER(C.c_uint32)]),
    "lr_server_preload": (C.c_int, [_vp, _u32]),
    "lr_server_submit_render": (C.c_int, [_vp, _u32, C.POINTER(Settings), C.POINTER(Frame), C.POINTER(C.c_float),
                                          C.POINTER(C.c_uint64)]),
    "lr_server_submit_probe": (C.c_int, [_vp, _u32, C.POINTER(Frame), _u32, C.POINTER(C.c_uint32),
                                         C.POINTER(C.c_float), C.POINTER(C.c_uint64)]),
    "lr_server_request_info": (C.c_int, [_vp, _u64, C.POINTER(RequestInfo)]),
    "lr_server_wait": (C.c_int, [_vp, _u64, C.c_double]),
    "lr_server_stats_get": (C.c_int, [_vp, C.POINTER(ServerStats)]),
    "lr_server_destroy": (None, [_vp]),
}

def exported_symbols() -> list[str]:
    """The entry points this harness binds (every one the header declares)."""
    return list(_SIGNATURES)


def _check(status: int) -> None:
    if status != 0:
        raise RenderError(status, (lib.lr_last_error() or b"").decode())


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _uptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _matrix12(m) -> "C.Array":
    arr = (C.c_double * 12)()
    if m is not None:
        arr[:] = [float(v) for v in np.asarray(m, np.float64).reshape(12)]
    return arr


# ---- context ----------------------------------------------------------------------------

class Context:
    """One CUDA device and stream (the reference's gpu.Device)."""

    def __init__(self, device: int = 0):
        handle = _vp()
        _check(lib.lr_context_create(device, C.byref(handle)))
        self.handle = handle
        self.device = device

    def synchronize(self) -> None:
        _check(lib.lr_context_synchronize(self.handle))

    def close(self) -> None:
        if self.handle:
            lib.lr_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # Device memory, for benches and tests that keep inputs resident in HBM.
    def alloc(self, nbytes: int) -> int:
        p = _vp()
        _check(lib.lr_device_alloc(self.handle, nbytes, C.byref(p)))
        return p.value

    def free(self, ptr: int) -> None:
        _check(lib.lr_device_free(self.handle, ptr))

    def upload(self, dst: int, array: np.ndarray) -> None:
        a = np.ascontiguousarray(array)
        _check(lib.lr_memcpy_htod(self.handle, dst, a.ctypes.data, a.nbytes))

    def download(self, src: int, out: np.ndarray) -> np.ndarray:
        _check(lib.lr_memcpy_dtoh(self.handle, out.ctypes.data, src, out.nbytes))
        return out

    def memset(self, dst: int, value: int, nbytes: int) -> None:
        _check(lib.lr_memset_device(self.handle, dst, value, nbytes))

    def memory(self, reset_high: bool = False) -> dict:
        """The device's memory: free and total bytes, and the default stream-ordered
        pool's bytes in use now and at most since the last reset (`reset_high` resets
        that mark to the current use first)."""
        out = (C.c_uint64 * 4)()
        _check(lib.lr_context_memory(self.handle, 1 if reset_high else 0, out))
        return {"free": out[0], "total": out[1], "pool_used": out[2], "pool_high": out[3]}

    def launch_overhead(self, count: int, graph: bool) -> tuple[float, float]:
        """Microseconds a launch of `count` dependent empty launches costs (direct, or
        one CUDA graph): on the device, and on the host's clock."""
        out = (C.c_double * 2)()
        _check(lib.lr_launch_overhead(self.handle, count, 1 if graph else 0, out))
        return out[0], out[1]

    def timer_start(self) -> None:
        _check(lib.lr_timer_start(self.handle))

    def timer_stop(self) -> float:
        ms = C.c_float()
        _check(lib.lr_timer_stop(self.handle, C.byref(ms)))
        return ms.value


class PinnedArray:
    """A page-locked host buffer viewed as a numpy array."""

    def __init__(self, shape, dtype):
        dtype = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * dtype.itemsize
        p = _vp()
        _check(lib.lr_host_alloc_pinned(max(nbytes, 16), C.byref(p)))
        self.ptr = p.value
        buf = (C.c_char * max(nbytes, 16)).from_address(self.ptr)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    def close(self) -> None:
        if self.ptr:
            self.array = None
            lib.lr_host_free_pinned(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- scene description -----------------------------------------------------------------

class MeshData:
    """A mesh as flat arrays: the stand-in for a luce-geocore Mesh in a GeometrySet."""

    def __init__(self, positions, indices, faces=None, face_count: int = 0, normals=None,
                 normals_per_corner: bool = False, face_materials=None, transform=None):
        self.positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        self.indices = np.ascontiguousarray(indices, np.uint32).reshape(-1, 3)
        self.faces = None if faces is None else np.ascontiguousarray(faces, np.uint32).reshape(-1)
        self.face_count = int(face_count)
        self.normals = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        self.normals_per_corner = bool(normals_per_corner)
        self.face_materials = None if face_materials is None else np.ascontiguousarray(face_materials, np.uint32)
        self.transform = transform

    def to_c(self) -> Mesh:
        m = Mesh()
        m.positions = _fptr(self.positions)
        m.point_count = len(self.positions)
        m.indices = _uptr(self.indices)
        m.triangle_count = len(self.indices)
        if self.faces is not None:
            m.triangle_faces = _uptr(self.faces)
        m.face_count = self.face_count
        if self.normals is not None:
            m.normals = _fptr(self.normals)
            m.normals_per_corner = 1 if self.normals_per_corner else 0
        if self.face_materials is not None:
            m.face_materials = _uptr(self.face_materials)
        m.transform = _matrix12(self.transform)
        return m


def placement(position=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0), scale=(1.0, 1.0, 1.0)) -> np.ndarray:
    """A 12-double placement (columns x, y, z, translation): scale, then rotation about
    X, then Y, then Z (radians), then translation."""
    rx, ry, rz = rotation
    cx, sx, cy, sy, cz, sz = np.cos(rx), np.sin(rx), np.cos(ry), np.sin(ry), np.cos(rz), np.sin(rz)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    M = Rz @ Ry @ Rx @ np.diag(np.asarray(scale, np.float64))
    return np.concatenate([M[:, 0], M[:, 1], M[:, 2], np.asarray(position, np.float64)])


def camera(position, rotation=(0.0, 0.0, 0.0), projection: int = 0, focal_length: float = 50.0,
           horizontal_aperture: float = 36.0, f_stop: float = 0.0, focus_distance: float = 5.0,
           matrix=None) -> Camera:
    c = Camera()
    c.matrix = _matrix12(matrix if matrix is not None else placement(position, rotation))
    c.projection = projection
    c.focal_length = focal_length
    c.horizontal_aperture = horizontal_aperture
    c.f_stop = f_stop
    c.focus_distance = focus_distance
    return c


def light(shape: int, position=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0), color=(1.0, 1.0, 1.0),
          intensity: float = 1.0, exposure: float = 0.0, temperature: float = 0.0, width: float = 1.0,
          height: float = 1.0, radius: float = 0.5, angle: float = 0.0, normalize: bool = False,
          visible: bool = True, matrix=None, image=None) -> Light:
    """A UsdLux light. `image`, for a dome: its lat-long image as linear Rec.709 RGB,
    height x width x 3 (rows from the top), kept alive with the light."""
    l = Light()
    l.matrix = _matrix12(matrix if matrix is not None else placement(position, rotation))
    l.shape = shape
    l.color[:] = list(color)
    l.intensity, l.exposure, l.temperature = intensity, exposure, temperature
    l.width, l.height, l.radius, l.angle = width, height, radius, angle
    l.normalize = 1 if normalize else 0
    l.visible = 1 if visible else 0
    if image is not None:
        pixels = np.ascontiguousarray(image, np.float32)
        if pixels.ndim != 3 or pixels.shape[2] != 3:
            raise ValueError("a dome's image is height x width x 3")
        l.keep_image = pixels
        l.image = pixels.ctypes.data_as(C.POINTER(C.c_float))
        l.image_height, l.image_width = pixels.shape[0], pixels.shape[1]
    return l


class CompiledScene:
    """render.CompiledScene (scene.lucb:31-63): owned here, freed by close()."""

    def __init__(self, handle):
        self.handle = handle

    @property
    def info(self) -> SceneInfo:
        info = SceneInfo()
        _check(lib.lr_scene_info_get(self.handle, C.byref(info)))
        return info

    def triangle_count(self) -> int:
        return int(self.info.triangle_count)

    def point_count(self) -> int:
        return int(self.info.point_count)

    def arrays(self) -> dict:
        """Copies of the compiled arrays: positions, indices, faces, shading, nodes, order."""
        info = self.info
        ptrs = [_vp() for _ in range(6)]
        _check(lib.lr_scene_arrays(self.handle, *[C.byref(p) for p in ptrs]))
        T, P, N = int(info.triangle_count), int(info.point_count), int(info.node_count)

        def view(ptr, count, dtype):
            if count == 0 or not ptr.value:
                return np.zeros(0, dtype)
            dt = np.dtype(dtype)
            buf = (C.c_char * (count * dt.itemsize)).from_address(ptr.value)
            return np.frombuffer(buf, dtype=dt, count=count).copy()

        return {
            "positions": view(ptrs[0], P * 3, np.float32).reshape(-1, 3),
            "indices": view(ptrs[1], T * 3, np.uint32).reshape(-1, 3),
            "faces": view(ptrs[2], T, np.uint32),
            "shading": view(ptrs[3], T * 4, np.uint32).reshape(-1, 4),
            "nodes": view(ptrs[4], N, NODE_DTYPE),
            "order": view(ptrs[5], T, np.uint32),
        }

    def camera(self, index: int = -1) -> Camera:
        c = Camera()
        _check(lib.lr_scene_camera(self.handle, index, C.byref(c)))
        return c

    def move_points(self, positions) -> None:
        """Moves the compiled points (point_count x 3, world space, the scene's point
        order) with the triangles kept, and refits the BVH2 and flat normals in place."""
        p = np.ascontiguousarray(positions, np.float32).reshape(-1)
        _check(lib.lr_scene_move_points(self.handle, p.ctypes.data_as(C.POINTER(C.c_float)), C.c_uint64(len(p) // 3)))

    def close(self) -> None:
        if self.handle:
            lib.lr_scene_free(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def compile_scene(meshes: Sequence[MeshData], cameras: Sequence[Camera] = (), lights: Sequence[Light] = (),
                  materials: Sequence[OpenPbr] = (), trees: bool = True) -> CompiledScene:
    """render.compile_scene (scene.lucb:111-129). Without `trees` the host builds no BVH2 and
    the triangles keep the meshes' order: such a scene is for GpuScene.build."""
    cm = (Mesh * max(1, len(meshes)))(*[m.to_c() for m in meshes])
    cc = (Camera * max(1, len(cameras)))(*cameras)
    cl = (Light * max(1, len(lights)))(*lights)
    cmat = (OpenPbr * max(1, len(materials)))(*materials)
    handle = _vp()
    _check(lib.lr_scene_compile_ex(cm, len(meshes), cc, len(cameras), cl, len(lights), cmat, len(materials),
                                   0 if trees else COMPILE_NO_TREES, C.byref(handle)))
    return CompiledScene(handle)


def ray_frame(cam: Camera, width: int, height: int) -> Frame:
    """render.ray_frame (camera.lucb:57-76)."""
    f = Frame()
    _check(lib.lr_ray_frame(C.byref(cam), width, height, C.byref(f)))
    return f


def look_frame(position, forward, up, tan_half_height: float, width: int, height: int,
               orthographic: bool = False) -> Frame:
    """render.look_frame (camera.lucb:84-95)."""
    f = Frame()
    p, fw, u = ((C.c_double * 3)(*map(float, v)) for v in (position, forward, up))
    _check(lib.lr_look_frame(p, fw, u, float(tan_half_height), width, height, 1 if orthographic else 0,
                             C.byref(f)))
    return f


class GpuScene:
    """render.GpuScene (device.lucb:16-38)."""

    def __init__(self, handle, ctx: Context):
        self.handle = handle
        self.ctx = ctx

    @staticmethod
    def upload(ctx: Context, scene: CompiledScene) -> "GpuScene":
        handle = _vp()
        _check(lib.lr_gpu_scene_upload(ctx.handle, scene.handle, C.byref(handle)))
        return GpuScene(handle, ctx)

    @staticmethod
    def build(ctx: Context, scene: CompiledScene) -> "GpuScene":
        """GpuScene.upload(accelerate = true) (device.lucb:41-89): the scene's triangles with a
        linear BVH2 built on the device (lr_gpu_scene_build). Probes and ray queries only."""
        handle = _vp()
        _check(lib.lr_gpu_scene_build(ctx.handle, scene.handle, C.byref(handle)))
        return GpuScene(handle, ctx)

    def destroy(self) -> None:
        if self.handle:
            lib.lr_gpu_scene_destroy(self.handle)
            self.handle = None

    close = destroy

    def refit(self, ctx: "Context", positions, device: bool = False) -> None:
        """Moves the uploaded points and refits the scene's BVHs on the device: `positions`
        a host array (point_count x 3), or with `device` the address of device memory and
        the point count as a (pointer, count) pair."""
        if device:
            ptr, count = positions
            _check(lib.lr_gpu_scene_refit(ctx.handle, self.handle, C.c_void_p(ptr), C.c_uint64(count), REFIT_DEVICE))
            return
        p = np.ascontiguousarray(positions, np.float32).reshape(-1)
        _check(lib.lr_gpu_scene_refit(ctx.handle, self.handle, p.ctypes.data_as(C.c_void_p), C.c_uint64(len(p) // 3), 0))

    @property
    def info(self) -> GpuSceneInfo:
        info = GpuSceneInfo()
        _check(lib.lr_gpu_scene_info_get(self.handle, C.byref(info)))
        return info

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def probe(ctx: Context, scene: GpuScene, frame: Frame, reference: bool = False):
    """render.probe (device.lucb:138-160): per pixel (row-major from the top) the polygon
    hit (0xffffffff none) and its distance along the frame's unnormalized direction."""
    n = int(frame.width) * int(frame.height)
    faces = np.empty(n, np.uint32)
    distances = np.empty(n, np.float32)
    _check(lib.lr_probe(ctx.handle, scene.handle, C.byref(frame), TRACE_REFERENCE if reference else 0,
                        _uptr(faces), _fptr(distances)))
    return faces, distances


PROBE_STATIC_PIXELS = 1 << 21
ALBEDO_TABLE_SIZE = 17440


def albedo_tables(ctx: Context) -> np.ndarray:
    """The albedo tables the glossy lobes read (E_ggx 32 x 32, its average over mu,
    E_dielectric 16 x 32 x 32), as made on the device."""
    out = np.empty(ALBEDO_TABLE_SIZE, np.float32)
    _check(lib.lr_albedo_tables(ctx.handle, _fptr(out), out.size))
    return out



def probe_static(ctx: Context, scene: GpuScene, frame: Frame, reference: bool = False):
    """probe() staged through the library's static device scratch (no device allocation;
    at most PROBE_STATIC_PIXELS pixels; calls on one device must not overlap)."""
    n = int(frame.width) * int(frame.height)
    faces = np.empty(n, np.uint32)
    distances = np.empty(n, np.float32)
    _check(lib.lr_probe_static(ctx.handle, scene.handle, C.byref(frame), TRACE_REFERENCE if reference else 0,
                               _uptr(faces), _fptr(distances)))
    return faces, distances


TRACE_BVH = {0: 0, 2: 8, 4: 16, 8: 32}


def trace_rays(ctx: Context, scene: GpuScene, rays: np.ndarray, any_hit: bool = False,
               reference: bool = False, count: bool = False, width: int = 0) -> np.ndarray:
    """Closest (or any) hits of rays (n x 8 floats: origin, tmin, direction, tmax):
    n x 4 words (t, triangle id as int32, u, v). `width` picks the watertight path's BVH
    (2, 4 or 8; 0 the default)."""
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    hits = np.empty((len(rays), 4), np.float32)
    flags = (TRACE_ANY if any_hit else 0) | (TRACE_REFERENCE if reference else 0) | (TRACE_COUNT if count else 0)
    flags |= TRACE_BVH[width]
    _check(lib.lr_trace_rays(ctx.handle, scene.handle, _fptr(rays), len(rays), _fptr(hits), flags))
    return hits


def trace_counts(ctx: Context):
    """Interior visits and triangle tests of counted queries since the last call."""
    out = (C.c_uint64 * 2)()
    _check(lib.lr_trace_counts(ctx.handle, out))
    return int(out[0]), int(out[1])


def hit_ids(hits: np.ndarray) -> np.ndarray:
    """The triangle ids (int32, -1 none) of a hits array."""
    return hits.view(np.int32)[:, 1].copy()


# ---- the renderer ------------------------------------------------------------------------

class RenderSettings:
    """RenderSettings (integrator.lucb:42-85)."""

    def __init__(self, settings: Settings):
        self.c = settings

    @staticmethod
    def of(width: int, height: int, samples: int) -> "RenderSettings":
        s = Settings()
        lib.lr_settings_default(C.byref(s), width, height, samples)
        return RenderSettings(s)

    def __getattr__(self, name):
        return getattr(self.__dict__["c"], name)

    def __setattr__(self, name, value):
        if name == "c":
            self.__dict__["c"] = value
        elif name in ("background",):
            self.c.background[:] = list(value)
        else:
            setattr(self.c, name, value)


class Renderer:
    """render.Renderer (integrator.lucb:259-900)."""

    def __init__(self, handle, ctx: Context, width: int, height: int):
        self.handle = handle
        self.ctx = ctx
        self.width, self.height = width, height

    @staticmethod
    def create(ctx: Context, scene: CompiledScene, settings: RenderSettings, frame: Frame | None = None) -> "Renderer":
        handle = _vp()
        if frame is None:
            _check(lib.lr_renderer_create(ctx.handle, scene.handle, C.byref(settings.c), C.byref(handle)))
            w, h = settings.c.width, settings.c.height
        else:
            _check(lib.lr_renderer_create_viewed(ctx.handle, scene.handle, C.byref(settings.c), C.byref(frame),
                                                 C.byref(handle)))
            w, h = frame.width, frame.height
        return Renderer(handle, ctx, int(w), int(h))

    def advance(self) -> bool:
        more = C.c_int32()
        _check(lib.lr_renderer_advance(self.handle, C.byref(more)))
        return bool(more.value)

    def finish(self) -> None:
        _check(lib.lr_renderer_finish(self.handle))

    def samples_done(self) -> int:
        return int(lib.lr_renderer_samples_done(self.handle))

    def passes(self):
        """(passes recorded, passes finished, bands a sample)."""
        rec, fin, bands = C.c_uint64(), C.c_uint64(), C.c_uint32()
        _check(lib.lr_renderer_passes(self.handle, C.byref(rec), C.byref(fin), C.byref(bands)))
        return int(rec.value), int(fin.value), int(bands.value)

    def advance_one(self) -> bool:
        """Advance until one more pass has been queued (False when none is left)."""
        recorded = self.passes()[0]
        while True:
            more = self.advance()
            if self.passes()[0] > recorded:
                return True
            if not more:
                return False

    def join(self) -> None:
        """Order the context's stream after the passes queued so far (no wait)."""
        _check(lib.lr_renderer_join(self.handle))

    def wait(self) -> None:
        """Wait for the passes queued so far."""
        self.join()
        self.ctx.synchronize()

    def read_into(self, out: np.ndarray) -> np.ndarray:
        """Renderer.read into a caller's float32 array of height x width x 4."""
        if out.dtype != np.float32 or out.size != self.width * self.height * 4 or not out.flags.c_contiguous:
            raise RenderError(INVALID, "reading the image needs four floats a pixel")
        _check(lib.lr_renderer_read(self.handle, _fptr(out), out.size))
        return out

    def read_async(self, out: np.ndarray) -> None:
        """Queues a copy of the image as the pass launched last leaves it into `out` (float32,
        height x width x 4; pinned, e.g. a PinnedArray's, for the copy to overlap the
        passes after it) and returns at once; `out` is complete after read_wait()."""
        if out.dtype != np.float32 or out.size != self.width * self.height * 4 or not out.flags.c_contiguous:
            raise RenderError(INVALID, "reading the image needs four floats a pixel")
        _check(lib.lr_renderer_read_async(self.handle, _fptr(out), out.size))

    def read_wait(self) -> None:
        """Waits for every copy read_async queued."""
        _check(lib.lr_renderer_read_wait(self.handle))

    def read_ticket(self, out: np.ndarray) -> int:
        """read_async, returning a ticket for read_landed."""
        if out.dtype != np.float32 or out.size != self.width * self.height * 4 or not out.flags.c_contiguous:
            raise RenderError(INVALID, "reading the image needs four floats a pixel")
        t = C.c_uint64()
        _check(lib.lr_renderer_read_ticket(self.handle, _fptr(out), out.size, C.byref(t)))
        return int(t.value)

    def read_landed(self, ticket: int) -> bool:
        """Whether the copy with `ticket` (and every one before it) has arrived; never waits."""
        v = C.c_int32()
        _check(lib.lr_renderer_read_landed(self.handle, ticket, C.byref(v)))
        return bool(v.value)

    def restart(self, frame: Frame) -> None:
        """Renderer.restart (integrator.lucb:463): start over through `frame`."""
        _check(lib.lr_renderer_restart(self.handle, C.byref(frame)))
        self.width, self.height = int(frame.width), int(frame.height)

    def reload(self, scene: "CompiledScene", settings: "RenderSettings", frame: Frame | None = None) -> None:
        """Renderer.reload (integrator.lucb:491): the same geometry, other lights,
        materials or settings."""
        _check(lib.lr_renderer_reload(self.handle, scene.handle, C.byref(settings.c),
                                      C.byref(frame) if frame is not None else None))
        if frame is not None:
            self.width, self.height = int(frame.width), int(frame.height)

    def replace_scene(self, scene: "CompiledScene", settings: "RenderSettings", frame: Frame) -> None:
        """Renderer.replace_scene (integrator.lucb:543): new geometry."""
        _check(lib.lr_renderer_replace_scene(self.handle, scene.handle, C.byref(settings.c), C.byref(frame)))
        self.width, self.height = int(frame.width), int(frame.height)

    def refit(self, scene: "CompiledScene", frame: Frame | None = None) -> None:
        """The renderer's geometry with its points moved (`scene` after move_points): its
        upload refit on the device, its lights loaded again, the film started over."""
        _check(lib.lr_renderer_refit(self.handle, scene.handle, C.byref(frame) if frame is not None else None))
        if frame is not None:
            self.width, self.height = int(frame.width), int(frame.height)

    def display(self) -> int:
        """The device address of the rgba16f display image."""
        p = _vp()
        _check(lib.lr_renderer_display(self.handle, C.byref(p)))
        return p.value or 0

    def shown_size(self) -> tuple[int, int]:
        out = (C.c_uint32 * 2)()
        _check(lib.lr_renderer_shown_size(self.handle, out))
        return int(out[0]), int(out[1])

    def read_display(self) -> np.ndarray:
        """The display image copied to the host (float16, shown height x width x 4)."""
        w, h = self.shown_size()
        out = np.zeros((h, w, 4), np.float16)
        if w and h:
            _check(lib.lr_memcpy_dtoh(self.ctx.handle, out.ctypes.data_as(_vp), C.c_void_p(self.display()), out.nbytes))
        return out

    def set_display(self, exposure: float = 0.0, view: int = 0) -> None:
        _check(lib.lr_renderer_set_display(self.handle, exposure, view))

    def converged_pixels(self) -> int:
        """Renderer.converged_pixels: pixels adaptive sampling has stopped."""
        out = C.c_uint64()
        _check(lib.lr_renderer_converged_pixels(self.handle, C.byref(out)))
        return int(out.value)

    def image(self) -> int:
        """The device address of the rgba32f image."""
        p = _vp()
        _check(lib.lr_renderer_image(self.handle, C.byref(p)))
        return p.value

    def read(self) -> np.ndarray:
        out = np.empty((self.height, self.width, 4), np.float32)
        _check(lib.lr_renderer_read(self.handle, _fptr(out), out.size))
        return out

    def set_samples(self, samples: int) -> None:
        _check(lib.lr_renderer_set_samples(self.handle, samples))

    def kernel_times(self) -> np.ndarray:
        out = (C.c_double * 10)()
        _check(lib.lr_renderer_kernel_times(self.handle, out))
        return np.array(out[:])

    def stats(self) -> RenderStats:
        s = RenderStats()
        _check(lib.lr_renderer_stats(self.handle, C.byref(s)))
        return s

    def recorded_rays(self, round_: int, shadow: bool = False) -> tuple[np.ndarray, np.ndarray]:
        """The last pass's rays of round `round_` (settings.profile = 3) as the ray
        queries take them -- (n, 8) float32: origin, t_min 0, direction, t_max -- and the
        traversal's answers, (n, 4): closest (t, id bits, u, v) or shadow (1 blocked, 0
        clear, -1 not traced by the any-hit query)."""
        n = C.c_uint64()
        _check(lib.lr_renderer_recorded_rays(self.handle, round_, int(shadow), None, 0, C.byref(n)))
        out = np.empty((n.value, 12), np.float32)
        _check(lib.lr_renderer_recorded_rays(self.handle, round_, int(shadow), _fptr(out), out.size, C.byref(n)))
        rays = out[:, :8].copy()
        rays[:, 3] = 0.0  # the origin's w holds the path's tag; the queries start at t 0
        return rays, out[:, 8:].copy()

    def destroy(self) -> None:
        if self.handle:
            lib.lr_renderer_destroy(self.handle)
            self.handle = None

    close = destroy

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Batch:
    """Many renders in one wavefront (lr_batch): members join with a GPU scene, the
    compiled scene it came from, RenderSettings and an optional frame, and each comes out
    as the image a Renderer of its own would make."""

    def __init__(self, ctx: Context, settings: BatchSettings | None = None):
        self.ctx = ctx
        self.handle = None
        self.sizes = {}
        h = _vp()
        _check(lib.lr_batch_create(ctx.handle, C.byref(settings or BatchSettings.default()), C.byref(h)))
        self.handle = h

    def add(self, gpu_scene: GpuScene, scene: CompiledScene, settings: RenderSettings,
            frame: Frame | None = None) -> int:
        member = C.c_uint32()
        _check(lib.lr_batch_add(self.handle, gpu_scene.handle, scene.handle, C.byref(settings.c),
                                C.byref(frame) if frame is not None else None, C.byref(member)))
        if frame is not None:
            self.sizes[member.value] = (int(frame.height), int(frame.width))
        else:
            self.sizes[member.value] = (int(settings.c.height), int(settings.c.width))
        return int(member.value)

    def remove(self, member: int) -> None:
        _check(lib.lr_batch_remove(self.handle, member))
        self.sizes.pop(member, None)

    def advance(self) -> bool:
        more = C.c_int32()
        _check(lib.lr_batch_advance(self.handle, C.byref(more)))
        return bool(more.value)

    def finish(self) -> None:
        _check(lib.lr_batch_finish(self.handle))

    def join(self) -> None:
        """Waits for the passes in flight and retires them."""
        _check(lib.lr_batch_join(self.handle))

    def info(self, member: int):
        """(samples done, samples planned, samples asked for)."""
        d, p, n = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(lib.lr_batch_member_info(self.handle, member, C.byref(d), C.byref(p), C.byref(n)))
        return int(d.value), int(p.value), int(n.value)

    def samples_done(self, member: int) -> int:
        return self.info(member)[0]

    def set_samples(self, member: int, samples: int) -> None:
        _check(lib.lr_batch_set_samples(self.handle, member, samples))

    def tune(self) -> dict:
        """Autotune, per scene-size class, BVH width, traversal stack depth and threads a
        block, then paths a pass, the interval of octant sorts of outgoing rays and the
        traversal warps' refill point, on the members as they stand (images do not
        change)."""
        t = BatchTuning()
        _check(lib.lr_batch_tune(self.handle, C.byref(t)))
        return {"width": int(t.width), "fill": int(t.fill), "paths_per_ms": float(t.paths_per_ms),
                "candidates": int(t.candidates), "class_width": list(t.class_width),
                "class_members": list(t.class_members), "class_stack": list(t.class_stack),
                "class_block": list(t.class_block), "bin_interval": int(t.bin_interval),
                "refill_at": int(t.refill_at), "thin_from": int(t.thin_from)}

    def passes(self):
        rec, fin = C.c_uint64(), C.c_uint64()
        _check(lib.lr_batch_passes(self.handle, C.byref(rec), C.byref(fin)))
        return int(rec.value), int(fin.value)

    def image(self, member: int) -> int:
        p = _vp()
        _check(lib.lr_batch_image(self.handle, member, C.byref(p)))
        return p.value

    def read(self, member: int) -> np.ndarray:
        h, w = self.sizes[member]
        out = np.empty((h, w, 4), np.float32)
        _check(lib.lr_batch_read(self.handle, member, _fptr(out), out.size))
        return out

    def read_into(self, member: int, out: np.ndarray) -> np.ndarray:
        if out.dtype != np.float32 or not out.flags.c_contiguous:
            raise RenderError(INVALID, "reading the image needs four floats a pixel")
        _check(lib.lr_batch_read(self.handle, member, _fptr(out), out.size))
        return out

    def read_async(self, member: int, out: np.ndarray) -> None:
        """Renderer.read_async for a member."""
        if out.dtype != np.float32 or not out.flags.c_contiguous:
            raise RenderError(INVALID, "reading the image needs four floats a pixel")
        _check(lib.lr_batch_read_async(self.handle, member, _fptr(out), out.size))

    def read_wait(self) -> None:
        _check(lib.lr_batch_read_wait(self.handle))

    def read_ticket(self, member: int, out: np.ndarray) -> int:
        """read_async, returning a ticket for read_landed."""
        if out.dtype != np.float32 or not out.flags.c_contiguous:
            raise RenderError(INVALID, "reading the image needs four floats a pixel")
        t = C.c_uint64()
        _check(lib.lr_batch_read_ticket(self.handle, member, _fptr(out), out.size, C.byref(t)))
        return int(t.value)

    def read_landed(self, ticket: int) -> bool:
        """Whether the copy with `ticket` (and every one before it) has arrived; never waits."""
        v = C.c_int32()
        _check(lib.lr_batch_read_landed(self.handle, ticket, C.byref(v)))
        return bool(v.value)

    def kernel_times(self) -> np.ndarray:
        out = (C.c_double * 10)()
        _check(lib.lr_batch_kernel_times(self.handle, out))
        return np.array(out[:])

    def stats(self) -> RenderStats:
        s = RenderStats()
        _check(lib.lr_batch_stats(self.handle, C.byref(s)))
        return s

    def destroy(self) -> None:
        if self.handle:
            lib.lr_batch_destroy(self.handle)
            self.handle = None

    close = destroy

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


REQUEST_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed"}


class Server:
    """The serving loop (lr_server): render sessions and probe queries submitted at any
    time, admitted by slots and memory budget, advanced together on one GPU."""

    def __init__(self, settings: ServerSettings | None = None):
        self.handle = None
        self._keep = {}    # buffers and scenes the library holds pointers to
        self._scenes = []
        h = _vp()
        _check(lib.lr_server_create(C.byref(settings or ServerSettings.default()), C.byref(h)))
        self.handle = h

    def add_scene(self, scene: CompiledScene) -> int:
        sid = C.c_uint32()
        _check(lib.lr_server_add_scene(self.handle, scene.handle, C.byref(sid)))
        self._scenes.append(scene)
        return int(sid.value)

    def preload(self, scene_id: int) -> None:
        _check(lib.lr_server_preload(self.handle, scene_id))

    def submit_render(self, scene_id: int, settings: RenderSettings, frame: Frame | None = None,
                      rgba: np.ndarray | None = None) -> int:
        if rgba is not None and (rgba.dtype != np.float32 or not rgba.flags.c_contiguous):
            raise RenderError(INVALID, "an image buffer is contiguous float32")
        rid = C.c_uint64()
        _check(lib.lr_server_submit_render(self.handle, scene_id, C.byref(settings.c),
                                           C.byref(frame) if frame is not None else None,
                                           _fptr(rgba) if rgba is not None else None, C.byref(rid)))
        if rgba is not None:
            self._keep[int(rid.value)] = (rgba,)
        return int(rid.value)

    def submit_probe(self, scene_id: int, frame: Frame, faces: np.ndarray, distances: np.ndarray,
                     reference: bool = False) -> int:
        n = int(frame.width) * int(frame.height)
        if faces.dtype != np.uint32 or distances.dtype != np.float32 or faces.size < n or distances.size < n:
            raise RenderError(INVALID, "a probe needs one result per pixel")
        rid = C.c_uint64()
        _check(lib.lr_server_submit_probe(self.handle, scene_id, C.byref(frame), TRACE_REFERENCE if reference else 0,
                                          _uptr(faces), _fptr(distances), C.byref(rid)))
        self._keep[int(rid.value)] = (faces, distances)
        return int(rid.value)

    def info(self, request: int) -> dict:
        i = RequestInfo()
        _check(lib.lr_server_request_info(self.handle, request, C.byref(i)))
        return {"kind": "probe" if i.kind == 1 else "render", "state": REQUEST_STATES.get(i.state, "?"),
                "status": int(i.status), "scene": int(i.scene), "pixels": int(i.pixels), "samples": int(i.samples),
                "samples_done": int(i.samples_done), "submitted": i.submitted, "admitted": i.admitted,
                "first": i.first, "finished": i.finished}

    def wait(self, request: int, timeout: float = 600.0) -> None:
        _check(lib.lr_server_wait(self.handle, request, float(timeout)))
        self._keep.pop(request, None)

    def stats(self) -> dict:
        s = ServerStats()
        _check(lib.lr_server_stats_get(self.handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in ServerStats._fields_}

    def destroy(self) -> None:
        if self.handle:
            lib.lr_server_destroy(self.handle)
            self.handle = None
            self._keep.clear()

    close = destroy

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


KERNEL_NAMES = ["camera", "intersect closest", "shade surface", "shade miss", "intersect shadow",
                "light emission", "finish", "film convert", "adaptive", "later rounds"]
