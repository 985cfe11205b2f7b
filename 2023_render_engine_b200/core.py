"""Python face of the C ABI: Context and Scene objects over librt_b200.so.

Device buffers are torch CUDA tensors (their data pointers go straight to the C ABI);
host buffers are numpy arrays. Nothing here computes: every call runs on the GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N


def _ptr(a) -> int | None:
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


class Context:
    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        N.check(N.lib().rt_context_create(device, ctypes.byref(h)))
        self.handle = h
        self.device = device

    def set_stream(self, stream_ptr: int):
        N.check(N.lib().rt_context_set_stream(self.handle, ctypes.c_void_p(stream_ptr)))

    def synchronize(self):
        N.check(N.lib().rt_context_synchronize(self.handle))

    def close(self):
        if self.handle:
            N.lib().rt_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """Scene container; mirrors Scene::build (integration/Scene.cu:56-95) + intersects."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = ctypes.c_void_p()
        N.check(N.lib().rt_scene_create(ctx.handle, ctypes.byref(h)))
        self.handle = h

    def add_mesh(self, vertices, indices, material: int = 0, shape_id: int = 0, transparent: bool = False,
                 normals=None, normal_indices=None) -> int:
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        i = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1, 3)
        nrm = None if normals is None else np.ascontiguousarray(normals, dtype=np.float32).reshape(-1, 3)
        nid = None if normal_indices is None else np.ascontiguousarray(normal_indices, dtype=np.uint32).reshape(-1, 3)
        first = ctypes.c_uint32()
        N.check(N.lib().rt_scene_add_mesh(self.handle, _ptr(v), v.shape[0], _ptr(i), i.shape[0], _ptr(nrm),
                                          0 if nrm is None else nrm.shape[0], _ptr(nid), material, shape_id,
                                          int(transparent), ctypes.byref(first)))
        return first.value

    def add_sphere(self, object_to_world, world_to_object, radius: float, material: int = 0, shape_id: int = 0,
                   transparent: bool = False) -> int:
        o2w = np.ascontiguousarray(object_to_world, dtype=np.float32).reshape(16)
        w2o = np.ascontiguousarray(world_to_object, dtype=np.float32).reshape(16)
        idx = ctypes.c_uint32()
        N.check(N.lib().rt_scene_add_sphere(self.handle, _ptr(o2w), _ptr(w2o), float(radius), material, shape_id,
                                            int(transparent), ctypes.byref(idx)))
        return idx.value

    def commit(self):
        N.check(N.lib().rt_scene_commit(self.handle))

    def stats(self) -> dict:
        s = N.SceneStats()
        N.check(N.lib().rt_scene_stats_get(self.handle, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in N.SceneStats._fields_}

    def trace_stats(self) -> dict:
        s = N.TraceStats()
        N.check(N.lib().rt_trace_stats_get(self.handle, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in N.TraceStats._fields_}

    # ---- tracing ----
    def trace_closest(self, rays_dev, hits_dev, n: int | None = None, flags: int = 0):
        """rays_dev: CUDA tensor of n*8 float32 (rt_ray); hits_dev: n*4 (rt_hit)."""
        if n is None:
            n = rays_dev.numel() // 8
        N.check(N.lib().rt_trace_closest(self.handle, rays_dev.data_ptr(), n, hits_dev.data_ptr(), flags))

    def trace_closest_host(self, rays: np.ndarray, flags: int = 0) -> np.ndarray:
        r = np.ascontiguousarray(rays)
        assert r.dtype == N.RAY_DTYPE
        hits = np.zeros(r.shape[0], dtype=N.HIT_DTYPE)
        N.check(N.lib().rt_trace_closest_host(self.handle, r.ctypes.data, r.shape[0], hits.ctypes.data, flags))
        return hits

    def trace_any(self, rays_dev, occluded_dev, n: int | None = None, flags: int = 0):
        if n is None:
            n = rays_dev.numel() // 8
        N.check(N.lib().rt_trace_any(self.handle, rays_dev.data_ptr(), n, occluded_dev.data_ptr(), flags))

    def close(self):
        if self.handle:
            N.lib().rt_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_rays(o: np.ndarray, d: np.ndarray, tmax=None) -> np.ndarray:
    """Packs origins/directions (n,3) into rt_ray records."""
    n = o.shape[0]
    r = np.zeros(n, dtype=N.RAY_DTYPE)
    r["ox"], r["oy"], r["oz"] = o[:, 0], o[:, 1], o[:, 2]
    r["dx"], r["dy"], r["dz"] = d[:, 0], d[:, 1], d[:, 2]
    r["tmax"] = np.inf if tmax is None else tmax
    return r
