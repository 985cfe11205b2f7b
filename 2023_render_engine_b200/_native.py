"""ctypes binding of the C ABI in include/rt_b200.h (librt_b200.so, built in-tree).

This is a thin loader: every function here forwards to the CUDA library. There is
no CPU fallback: if the library is missing, import fails loudly.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
# RT_B200_LIB overrides the library path (A/B comparisons of builds)
LIB_PATH = Path(os.environ["RT_B200_LIB"]) if os.environ.get("RT_B200_LIB") else _HERE / "lib" / "librt_b200.so"

RT_OK = 0
RT_TRACE_SHADOW = 0x1
RT_TRACE_FAST = 0x2
RT_TRACE_COUNT_ANY = 0x4
RT_PRIM_SHAPE = 0x40000000

STATUS_NAMES = {0: "RT_OK", 1: "RT_ERR_INVALID", 2: "RT_ERR_CUDA", 3: "RT_ERR_OOM", 4: "RT_ERR_TIMEOUT",
                5: "RT_ERR_UNSUPPORTED", 6: "RT_ERR_STATE", 7: "RT_ERR_CAPACITY"}

RAY_DTYPE = np.dtype([("ox", "<f4"), ("oy", "<f4"), ("oz", "<f4"), ("tmax", "<f4"),
                      ("dx", "<f4"), ("dy", "<f4"), ("dz", "<f4"), ("flags", "<u4")], align=True)
HIT_DTYPE = np.dtype([("t", "<f4"), ("prim", "<i4"), ("b1", "<f4"), ("b2", "<f4")], align=True)


class RtError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class SceneStats(ctypes.Structure):
    _fields_ = [("triangles", ctypes.c_uint64), ("spheres", ctypes.c_uint64), ("bvh8_nodes", ctypes.c_uint64),
                ("bvh8_leaf_triangles", ctypes.c_uint64), ("device_bytes", ctypes.c_uint64),
                ("build_ms", ctypes.c_double)]


class Material(ctypes.Structure):
    _fields_ = [("type", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("color", ctypes.c_float * 3),
                ("intensity", ctypes.c_float), ("eta", ctypes.c_float * 3), ("k", ctypes.c_float * 3),
                ("roughness", ctypes.c_float * 2), ("ior", ctypes.c_float), ("extra", ctypes.c_float * 3),
                ("texture", ctypes.c_uint32)]


class Camera(ctypes.Structure):
    _fields_ = [("camera_to_world", ctypes.c_float * 16), ("raster_to_camera", ctypes.c_float * 16),
                ("lens_radius", ctypes.c_float), ("focal_distance", ctypes.c_float),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32)]


class RenderOpts(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_uint32), ("sample_offset", ctypes.c_uint32), ("max_depth", ctypes.c_uint32),
                ("rr_depth", ctypes.c_uint32), ("seed", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("max_paths", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class View(ctypes.Structure):
    _fields_ = [("camera", Camera), ("spp", ctypes.c_uint32), ("sample_offset", ctypes.c_uint32),
                ("max_depth", ctypes.c_uint32), ("rr_depth", ctypes.c_uint32), ("seed", ctypes.c_uint32),
                ("scene", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 2)]


class RenderStats(ctypes.Structure):
    _fields_ = [("camera_rays", ctypes.c_uint64), ("extension_rays", ctypes.c_uint64),
                ("shadow_rays", ctypes.c_uint64), ("waves", ctypes.c_uint64), ("ms", ctypes.c_double),
                ("gathers", ctypes.c_uint64)]


RT_MAT_LAMBERTIAN, RT_MAT_TROWBRIDGE, RT_MAT_DIELECTRIC, RT_MAT_LIGHT, RT_MAT_MIRROR, RT_MAT_PLAIN = range(6)
RT_MAT_BECKMANN, RT_MAT_TROWBRIDGE_BASIC, RT_MAT_FRESNEL_BLEND, RT_MAT_PLASTIC = 8, 9, 10, 11
RT_MAT_PHONG = 6
RT_MAT_SUBSURFACE = 7
RT_MATF_TRANSPARENT = 0x1
RT_RENDER_NEE_AREA = 0x1
RT_RENDER_COMPAT = 0x2
RT_RENDER_EXACT_TRACE = 0x4
RT_RENDER_PHOTON_MAP = 0x8
RT_RENDER_GUIDE = 0x10
RT_RENDER_STAGE_TIMES = 0x100
RENDER_STAGES = ("trace", "guide_inference", "material_sort", "shade", "shadow", "gather", "retire")
RT_BUILD_DEVICE, RT_BUILD_HOST = 0, 1
(RT_TONEMAP_EQUALIZE, RT_TONEMAP_REINHARD, RT_TONEMAP_REINHARD_JODIE, RT_TONEMAP_ACES, RT_TONEMAP_UNCHARTED2,
 RT_TONEMAP_GAMMA_CLAMP) = range(6)
RT_RENDER_SUBSURFACE = 0x20
RT_RENDER_HYBRID = 0x40
RT_RENDER_HOST_LOOP = 0x80


class PhotonTraceStats(ctypes.Structure):
    _fields_ = [("emitted", ctypes.c_uint64), ("stored", ctypes.c_uint64), ("rays", ctypes.c_uint64),
                ("ms", ctypes.c_double)]


PHOTON_DTYPE = np.dtype([("pos", "<f4", 3), ("shape_id", "<i4"), ("dir", "<f4", 3), ("path", "<u4"),
                         ("power", "<f4", 3), ("depth", "<u4"), ("normal", "<f4", 3), ("reserved", "<f4")])


class GuideOpts(ctypes.Structure):
    _fields_ = [("bbox_min", ctypes.c_float * 3), ("bbox_max", ctypes.c_float * 3), ("learning_rate", ctypes.c_float),
                ("seed", ctypes.c_uint32), ("record_capacity", ctypes.c_uint32), ("max_depth", ctypes.c_uint32)]


GUIDE_INPUTS = 144
GUIDE_OUTPUTS = 48
GUIDE_LOBES = 8


class TraceStats(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_uint64), ("exact_fallback_rays", ctypes.c_uint64)]


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_I32 = ctypes.c_int32
_INT = ctypes.c_int
_F32 = ctypes.c_float

# name -> argtypes (all return int status)
SIGNATURES = {
    "rt_abi_version": [],
    "rt_last_error": [ctypes.c_char_p, ctypes.c_size_t],
    "rt_context_create": [_INT, ctypes.POINTER(_P)],
    "rt_context_destroy": [_P],
    "rt_context_set_stream": [_P, _P],
    "rt_context_synchronize": [_P],
    "rt_scene_create": [_P, ctypes.POINTER(_P)],
    "rt_scene_destroy": [_P],
    "rt_scene_add_mesh": [_P, _P, _U32, _P, _U32, _P, _U32, _P, _U32, _I32, _INT, ctypes.POINTER(_U32)],
    "rt_scene_add_sphere": [_P, _P, _P, _F32, _U32, _I32, _INT, ctypes.POINTER(_U32)],
    "rt_scene_add_plane": [_P, _P, _P, _U32, _I32, _INT, ctypes.POINTER(_U32)],
    "rt_scene_commit": [_P],
    "rt_scene_set_build": [_P, _U32],
    "rt_material_eval": [_P, _P, _P, ctypes.c_uint64, _P, _P],
    "rt_material_sample": [_P, _P, ctypes.c_uint64, _U32, _U32, _P, _P, _P, _P],
    "rt_film_tonemap": [_P, _P, _P, ctypes.c_uint64, ctypes.c_uint64, _U32, _P],
    "rt_image_write_bmp": [ctypes.c_char_p, _P, _U32, _U32],
    "rt_image_write_ppm": [ctypes.c_char_p, _P, _U32, _U32],
    "rt_scene_export_bvh": [_P, _P, _P, _P, _P, _P, _P],
    "rt_scene_stats_get": [_P, ctypes.POINTER(SceneStats)],
    "rt_trace_closest": [_P, _P, _U64, _P, _U32],
    "rt_trace_closest_host": [_P, _P, _U64, _P, _U32],
    "rt_trace_closest_noalloc": [_P, _P, _U64, _P, _U32],
    "rt_trace_any": [_P, _P, _U64, _P, _U32],
    "rt_trace_any_bits": [_P, _P, _U64, _P, _U32],
    "rt_trace_counts": [_P, _P, _U64, _U32, _P],
    "rt_render_stage_times": [_P, _P, _U32],
    "rt_trace_stats_get": [_P, ctypes.POINTER(TraceStats)],
    "rt_scene_set_materials": [_P, _P, _U32],
    "rt_scene_set_triangle_materials": [_P, _U32, _U32, _P],
    "rt_scene_add_texture": [_P, _P, _U32, _U32, _P],
    "rt_material_single_scattering": [_P, _P, _P, _P, _U64, _P, _P, _P],
    "rt_scene_set_triangle_uvs": [_P, _U32, _U32, _P],
    "rt_texture_lookup": [_P, _U32, _P, _U64, _P],
    "rt_scene_add_point_light": [_P, _P, _P, _F32],
    "rt_render": [_P, ctypes.POINTER(Camera), ctypes.POINTER(RenderOpts), _P, _P, _P, ctypes.POINTER(RenderStats)],
    "rt_render_set_sort": [_P, _U32],
    "rt_scene_merge": [_P, _P, _U32, ctypes.POINTER(_P)],
    "rt_render_batch": [_P, ctypes.POINTER(View), _U32, _U32, _U32, _P, _P, _P, ctypes.POINTER(RenderStats)],
    "rt_film_store_hdrbmp": [ctypes.c_char_p, _U32, _U32, _P, _P, _P, _U64],
    "rt_film_load_hdrbmp": [ctypes.c_char_p, _U32, _U32, _P, ctypes.POINTER(_U64)],
    "rt_film_rmse": [_P, _P, _P, _P, _P, _P, _U64, ctypes.POINTER(ctypes.c_double)],
    "rt_photons_trace": [_P, _U64, _U32, _U32, _U32, _U32, ctypes.POINTER(_P), ctypes.POINTER(PhotonTraceStats)],
    "rt_photon_map_from_points": [_P, _P, _P, _U64, ctypes.POINTER(_P)],
    "rt_photon_map_build": [_P],
    "rt_photon_map_count": [_P, ctypes.POINTER(_U64)],
    "rt_photon_map_get": [_P, _U64, _U64, _P],
    "rt_photon_map_destroy": [_P],
    "rt_photon_knn": [_P, _P, _P, _U64, _U32, _F32, _P, _P, _P],
    "rt_photon_density": [_P, ctypes.POINTER(Material), _P, _P, _P, _P, _U64, _U32, _F32, _P],
    "rt_photon_subsurface": [_P, ctypes.POINTER(Material), _P, _P, _P, _P, _U64, _F32, _U32, _P],
    "rt_render_set_photon_map": [_P, _P, _U32, _F32],
    "rt_guide_create": [_P, ctypes.POINTER(GuideOpts), ctypes.POINTER(_P)],
    "rt_guide_destroy": [_P],
    "rt_guide_param_count": [_P, ctypes.POINTER(_U64)],
    "rt_guide_params_get": [_P, _P, _U64],
    "rt_guide_params_set": [_P, _P, _U64],
    "rt_guide_steps": [_P, ctypes.POINTER(_U64)],
    "rt_guide_reset": [_P],
    "rt_guide_eval": [_P, _P, _U64, _P],
    "rt_guide_pdf": [_P, _P, _P, _P, _U64, _P],
    "rt_guide_sample": [_P, _P, _P, _U64, _P, _P],
    "rt_guide_train_step": [_P, _P, _P, _P, _P, _U64, _INT, _P, ctypes.POINTER(_F32)],
    "rt_render_set_guide": [_P, _P, _INT],
    "rt_guide_record_count": [_P, ctypes.POINTER(_U64), ctypes.POINTER(_U64)],
    "rt_guide_train_records": [_P, _U32, _U32, _U32, ctypes.POINTER(_F32)],
    "rt_guide_records_get": [_P, _U64, _U64, _P],
}


def load(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"CUDA core library not built: {p} (run __graft_entry__.build())")
    lib = ctypes.CDLL(str(p))
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    return lib


_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = load()
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().rt_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int):
    if status != RT_OK:
        raise RtError(status, last_error())
