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

    def __init__(self, ctx: Context, handle=None):
        self.ctx = ctx
        if handle is None:
            handle = ctypes.c_void_p()
            N.check(N.lib().rt_scene_create(ctx.handle, ctypes.byref(handle)))
        self.handle = handle

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

    def add_plane(self, object_to_world, world_to_object, material: int = 0, shape_id: int = 0,
                  transparent: bool = False) -> int:
        """rt_scene_add_plane: the unit square of the plane's object space (Plane.cu); returns its
        shape index (shared with spheres, in the order they are added)."""
        o2w = np.ascontiguousarray(object_to_world, dtype=np.float32).reshape(16)
        w2o = np.ascontiguousarray(world_to_object, dtype=np.float32).reshape(16)
        idx = ctypes.c_uint32()
        N.check(N.lib().rt_scene_add_plane(self.handle, _ptr(o2w), _ptr(w2o), material, shape_id, int(transparent),
                                           ctypes.byref(idx)))
        return idx.value

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

    def set_build(self, mode: int):
        """Where commit() builds: N.RT_BUILD_DEVICE (default) or N.RT_BUILD_HOST (same bytes)."""
        N.check(N.lib().rt_scene_set_build(self.handle, mode))

    def export_bvh(self):
        """The committed structures: (nodes (k, 80) uint8, records (n, 12) float32 whose w lanes
        hold rank / triangle id / flags bits, reference-tree boxes (2n - 1, 6) float32)."""
        nn, nr, nb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        N.check(N.lib().rt_scene_export_bvh(self.handle, None, None, None, ctypes.byref(nn), ctypes.byref(nr),
                                            ctypes.byref(nb)))
        nodes = np.zeros((nn.value, 80), np.uint8)
        recs = np.zeros((nr.value, 12), np.float32)
        boxes = np.zeros((nb.value, 6), np.float32)
        N.check(N.lib().rt_scene_export_bvh(self.handle, nodes.ctypes.data if nodes.size else None,
                                            recs.ctypes.data if recs.size else None,
                                            boxes.ctypes.data if boxes.size else None, ctypes.byref(nn),
                                            ctypes.byref(nr), ctypes.byref(nb)))
        return nodes, recs, boxes

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
        """Scene::isVisible's occlusion: occluded_dev gets one byte per ray (1: something is hit
        no farther than the ray's tmax)."""
        if n is None:
            n = rays_dev.numel() // 8
        N.check(N.lib().rt_trace_any(self.handle, rays_dev.data_ptr(), n, occluded_dev.data_ptr(), flags))

    def trace_any_bits(self, rays_dev, bits_dev, n: int | None = None, flags: int = 0):
        """The same decisions as a bit mask: ray i is bit i % 32 of 32-bit word i // 32."""
        if n is None:
            n = rays_dev.numel() // 8
        N.check(N.lib().rt_trace_any_bits(self.handle, rays_dev.data_ptr(), n, bits_dev.data_ptr(), flags))

    def trace_counts(self, rays_dev, counts_dev, n: int | None = None, flags: int = 0):
        """Traversal work per ray: counts_dev (2n int32) gets, for ray i, the BVH8 nodes visited
        (80 B each) and the triangle records tested (48 B each) by the closest-hit walk, or by
        the any-hit walk with N.RT_TRACE_COUNT_ANY."""
        if n is None:
            n = rays_dev.numel() // 8
        N.check(N.lib().rt_trace_counts(self.handle, rays_dev.data_ptr(), n, flags, counts_dev.data_ptr()))

    # ---- rendering ----
    def set_materials(self, mats):
        arr = (N.Material * len(mats))(*mats)
        N.check(N.lib().rt_scene_set_materials(self.handle, ctypes.cast(arr, ctypes.c_void_p), len(mats)))

    def set_triangle_materials(self, first: int, mat_ids):
        m = np.ascontiguousarray(mat_ids, dtype=np.uint32)
        N.check(N.lib().rt_scene_set_triangle_materials(self.handle, first, m.shape[0], m.ctypes.data))

    def add_texture(self, rgb) -> int:
        """rgb: (height, width, 3) texels, rows in Texture::pixelMatrix order. Returns the id."""
        a = np.ascontiguousarray(rgb, dtype=np.float32)
        if a.ndim != 3 or a.shape[2] != 3:
            raise ValueError("texture must be (height, width, 3)")
        tid = ctypes.c_uint32()
        N.check(N.lib().rt_scene_add_texture(self.handle, a.ctypes.data, a.shape[1], a.shape[0], ctypes.byref(tid)))
        return tid.value

    def set_triangle_uvs(self, first: int, uv):
        """uv: (n, 3, 2) texture coordinates of triangles [first, first + n)."""
        a = np.ascontiguousarray(uv, dtype=np.float32).reshape(-1, 6)
        N.check(N.lib().rt_scene_set_triangle_uvs(self.handle, first, a.shape[0], a.ctypes.data))

    def texture_lookup(self, tid: int, uv_dev):
        """Texture::getColor of texture tid at the (n, 2) device points; returns (n, 3)."""
        import torch

        n = uv_dev.numel() // 2
        out = torch.empty(3 * n, dtype=torch.float32, device=uv_dev.device)
        N.check(N.lib().rt_texture_lookup(self.handle, tid, uv_dev.data_ptr(), n, out.data_ptr()))
        return out.view(n, 3)

    def add_point_light(self, pos, rgb, intensity: float):
        p = np.ascontiguousarray(pos, dtype=np.float32)
        c = np.ascontiguousarray(rgb, dtype=np.float32)
        N.check(N.lib().rt_scene_add_point_light(self.handle, p.ctypes.data, c.ctypes.data, float(intensity)))

    def set_sort(self, chunk_log2: int):
        """Material sort of the wavefront's shading order in chunks of 2^chunk_log2 slots (0: off)."""
        N.check(N.lib().rt_render_set_sort(self.handle, int(chunk_log2)))

    def render(self, camera: "N.Camera", spp: int, max_depth: int, rr_depth: int = 3, seed: int = 0,
               flags: int = 0, sample_offset: int = 0, film=None, fp64: bool = False, max_paths: int = 0):
        """Adds spp samples per pixel into `film` (dict of torch tensors sum/count[/sum64]);
        returns (film, stats)."""
        import torch

        w, h = camera.width, camera.height
        if film is None:
            film = {"sum": torch.zeros(h * w * 3, dtype=torch.float32, device="cuda"),
                    "count": torch.zeros(h * w, dtype=torch.int32, device="cuda")}
            if fp64:
                film["sum64"] = torch.zeros(h * w * 3, dtype=torch.float64, device="cuda")
        opts = N.RenderOpts(spp, sample_offset, max_depth, rr_depth, seed, flags, max_paths, 0)
        st = N.RenderStats()
        s64 = film.get("sum64")
        N.check(N.lib().rt_render(self.handle, ctypes.byref(camera), ctypes.byref(opts), film["sum"].data_ptr(),
                                  film["count"].data_ptr(), None if s64 is None else s64.data_ptr(),
                                  ctypes.byref(st)))
        return film, {f: getattr(st, f) for f, _ in N.RenderStats._fields_}

    def stage_times(self) -> dict:
        """Per-stage device milliseconds of the last render made with N.RT_RENDER_STAGE_TIMES."""
        out = (ctypes.c_double * len(N.RENDER_STAGES))()
        N.check(N.lib().rt_render_stage_times(self.handle, out, len(N.RENDER_STAGES)))
        return dict(zip(N.RENDER_STAGES, list(out)))

    def render_batch(self, views, flags: int = 0, max_paths: int = 0, film=None, fp64: bool = False):
        """Renders many views of this scene in one wavefront (rt_render_batch).

        views: list of dicts with camera and spp, and optionally max_depth (8), rr_depth (3),
        seed (0), sample_offset (0), scene (0: the view's scene in a merged scene). The film holds
        the views' pixels back to back; returns (film, stats, offsets) with view i's pixels at
        [offsets[i], offsets[i + 1])."""
        import torch

        arr = (N.View * len(views))()
        offsets = [0]
        for i, v in enumerate(views):
            arr[i].camera = v["camera"]
            arr[i].spp = v["spp"]
            arr[i].sample_offset = v.get("sample_offset", 0)
            arr[i].max_depth = v.get("max_depth", 8)
            arr[i].rr_depth = v.get("rr_depth", 3)
            arr[i].seed = v.get("seed", 0)
            arr[i].scene = v.get("scene", 0)
            offsets.append(offsets[-1] + v["camera"].width * v["camera"].height)
        npx = offsets[-1]
        if film is None:
            film = {"sum": torch.zeros(npx * 3, dtype=torch.float32, device="cuda"),
                    "count": torch.zeros(npx, dtype=torch.int32, device="cuda")}
            if fp64:
                film["sum64"] = torch.zeros(npx * 3, dtype=torch.float64, device="cuda")
        st = N.RenderStats()
        s64 = film.get("sum64")
        N.check(N.lib().rt_render_batch(self.handle, arr, len(views), flags, max_paths, film["sum"].data_ptr(),
                                        film["count"].data_ptr(), None if s64 is None else s64.data_ptr(),
                                        ctypes.byref(st)))
        return film, {f: getattr(st, f) for f, _ in N.RenderStats._fields_}, offsets

    def set_photon_map(self, pmap, k: int = 100, radius: float = 100.0):
        """Photon map for RT_RENDER_PHOTON_MAP renders (MAX_NEIGHBOURS, PHOTON_SEARCH_RADIUS)."""
        N.check(N.lib().rt_render_set_photon_map(self.handle, None if pmap is None else pmap.handle, k,
                                                 float(radius)))
        self._pmap = pmap

    def set_guide(self, guide, train: bool = False):
        """Learned proposal for RT_RENDER_GUIDE renders; train=True records training samples."""
        N.check(N.lib().rt_render_set_guide(self.handle, None if guide is None else guide.handle, int(train)))
        self._guide = guide

    def trace_photons(self, n: int, max_depth: int = 30, rr_depth: int = 3, seed: int = 0, flags: int = 0):
        """Scene::generatePhotons + computePhotons: returns (PhotonMap, stats)."""
        h = ctypes.c_void_p()
        st = N.PhotonTraceStats()
        N.check(N.lib().rt_photons_trace(self.handle, n, max_depth, rr_depth, seed, flags, ctypes.byref(h),
                                         ctypes.byref(st)))
        # the map keeps the context alive, not the scene: a scene holding its photon map
        # (set_photon_map) would otherwise form a cycle whose finalisation order is arbitrary
        return PhotonMap(h, owner=self.ctx), {f: getattr(st, f) for f, _ in N.PhotonTraceStats._fields_}

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


def merge_scenes(ctx: Context, scenes) -> Scene:
    """rt_scene_merge: committed scenes of `ctx` as one scene whose render_batch views name their
    scene by its index in `scenes` (key "scene")."""
    arr = (ctypes.c_void_p * len(scenes))(*[s.handle.value if hasattr(s.handle, "value") else s.handle
                                           for s in scenes])
    h = ctypes.c_void_p()
    N.check(N.lib().rt_scene_merge(ctx.handle, ctypes.cast(arr, ctypes.c_void_p), len(scenes), ctypes.byref(h)))
    return Scene(ctx, handle=h)


def material(type_, color=(0.8, 0.8, 0.8), intensity=0.0, eta=(1.5, 1.5, 1.5), k=(0.0, 0.0, 0.0),
             roughness=(0.1, 0.1), ior=1.5, transparent=False, extra=(0.0, 0.0, 0.0), texture=None) -> "N.Material":
    """texture: a scene texture id (Scene.add_texture) or None."""
    m = N.Material()
    m.texture = 0 if texture is None else int(texture) + 1
    m.extra[:] = [float(c) for c in extra]
    m.type = type_
    m.flags = N.RT_MATF_TRANSPARENT if transparent else 0
    m.color[:] = [float(c) for c in color]
    m.intensity = float(intensity)
    m.eta[:] = [float(c) for c in eta]
    m.k[:] = [float(c) for c in k]
    m.roughness[:] = [float(c) for c in roughness]
    m.ior = float(ior)
    return m


def phong_material(kd, ks, ns, transparent=False) -> "N.Material":
    """PhongMaterial(ka, kd, ks, ke = 0, ni, ns) as the renderer's table entry."""
    return material(N.RT_MAT_PHONG, color=kd, k=ks, roughness=(ns, 0.0), transparent=transparent)


def subsurface_material(kd, ks, ns, eta, sigma_s, sigma_a, g=0.0, transparent=False) -> "N.Material":
    """SSMaterial(ka, kd, ks, eta, ns, texture, transparent, sigmaS, sigmaA, g)."""
    return material(N.RT_MAT_SUBSURFACE, color=kd, k=ks, roughness=(ns, g), ior=eta, eta=sigma_s, extra=sigma_a,
                    transparent=transparent)


def look_at_camera(eye, target, up, vfov_deg: float, width: int, height: int, focal=0.8,
                   lens_radius=0.0, focal_distance=1.0) -> "N.Camera":
    """Pinhole camera in the reference's convention: camera space looks along +z, the image
    plane at z = focal with half-height focal*tan(vfov/2) (an .obejota camera with
    cts = (0,0,-focal), frameY = 2*focal*tan(vfov/2)); raster y grows downwards."""
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    c2w = np.eye(4)
    c2w[:3, 0], c2w[:3, 1], c2w[:3, 2], c2w[:3, 3] = r, u, f, eye
    half_h = focal * np.tan(np.radians(vfov_deg) / 2)
    half_w = half_h * width / height
    # raster (x, y) -> camera (x', y', focal): x' = (x/W - 0.5) * 2 half_w, y' = (0.5 - y/H) * 2 half_h
    r2c = np.array([[2 * half_w / width, 0, 0, -half_w],
                    [0, -2 * half_h / height, 0, half_h],
                    [0, 0, 0, focal],
                    [0, 0, 0, 1]], np.float64)
    cam = N.Camera()
    cam.camera_to_world[:] = [float(x) for x in c2w.reshape(-1)]
    cam.raster_to_camera[:] = [float(x) for x in r2c.reshape(-1)]
    cam.lens_radius = float(lens_radius)
    cam.focal_distance = float(focal_distance)
    cam.width, cam.height = int(width), int(height)
    return cam


def film_mean(film) -> np.ndarray:
    """Per-pixel estimate sum / count as an (H*W, 3) float64 array."""
    s = (film["sum64"] if "sum64" in film else film["sum"]).double().cpu().numpy().reshape(-1, 3)
    c = film["count"].cpu().numpy().astype(np.float64)
    return s / np.maximum(c, 1)[:, None]


class PhotonMap:
    """Photon map handle: photons, kd-tree build, k-nearest gather (device buffers)."""

    def __init__(self, handle, owner=None):
        self.handle = handle
        self.owner = owner  # keeps the context (or the scene holding it) alive

    @classmethod
    def from_points(cls, ctx: Context, pos_dev, shape_dev=None):
        h = ctypes.c_void_p()
        n = pos_dev.numel() // 3
        N.check(N.lib().rt_photon_map_from_points(ctx.handle, pos_dev.data_ptr(),
                                                  None if shape_dev is None else shape_dev.data_ptr(), n,
                                                  ctypes.byref(h)))
        return cls(h, owner=ctx)

    def build(self):
        N.check(N.lib().rt_photon_map_build(self.handle))
        return self

    def __len__(self):
        n = ctypes.c_uint64()
        N.check(N.lib().rt_photon_map_count(self.handle, ctypes.byref(n)))
        return n.value

    def photons(self) -> np.ndarray:
        n = len(self)
        out = np.zeros(n, dtype=N.PHOTON_DTYPE)
        if n:
            N.check(N.lib().rt_photon_map_get(self.handle, 0, n, out.ctypes.data))
        return out

    def knn(self, queries_dev, k: int, radius: float, shape_dev=None, with_dist=True):
        import torch

        nq = queries_dev.numel() // 3
        idx = torch.empty(nq * k, dtype=torch.int32, device="cuda")
        dist = torch.empty(nq * k, dtype=torch.float32, device="cuda") if with_dist else None
        cnt = torch.empty(nq, dtype=torch.int32, device="cuda")
        N.check(N.lib().rt_photon_knn(self.handle, queries_dev.data_ptr(),
                                      None if shape_dev is None else shape_dev.data_ptr(), nq, k, float(radius),
                                      idx.data_ptr(), None if dist is None else dist.data_ptr(), cnt.data_ptr()))
        return idx.view(nq, k), (None if dist is None else dist.view(nq, k)), cnt

    def density(self, material: "N.Material", points_dev, normals_dev, wo_dev, k: int, radius: float,
                shape_dev=None):
        """Scene::combinePhotonContributions at each point; returns (nq, 3) CUDA tensor."""
        import torch

        nq = points_dev.numel() // 3
        out = torch.empty(nq * 3, dtype=torch.float32, device="cuda")
        N.check(N.lib().rt_photon_density(self.handle, ctypes.byref(material), points_dev.data_ptr(),
                                          normals_dev.data_ptr(), wo_dev.data_ptr(),
                                          None if shape_dev is None else shape_dev.data_ptr(), nq, k, float(radius),
                                          out.data_ptr()))
        return out.view(nq, 3)

    def close(self):
        if self.handle:
            N.lib().rt_photon_map_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def rmse(film_a, film_b) -> float:
    """computeRMSE (camera/Film.cu:611-632): sqrt(sum over pixels of |mean_a - mean_b|^2 / pixels),
    |.|^2 the squared norm of the RGB difference. Accepts films or (H*W, 3) arrays."""
    a = film_mean(film_a) if isinstance(film_a, dict) else np.asarray(film_a, dtype=np.float64).reshape(-1, 3)
    b = film_mean(film_b) if isinstance(film_b, dict) else np.asarray(film_b, dtype=np.float64).reshape(-1, 3)
    if a.shape != b.shape:
        return -1.0
    return float(np.sqrt(np.sum((a - b) ** 2) / a.shape[0]))


class Guide:
    """Learned path guide (vMF-mixture MLP): evaluation, training, parameters (device buffers)."""

    def __init__(self, ctx: Context, bbox_min, bbox_max, learning_rate: float = 1e-2, seed: int = 0,
                 record_capacity: int = 0, max_depth: int = 0):
        o = N.GuideOpts()
        for a in range(3):
            o.bbox_min[a] = float(bbox_min[a])
            o.bbox_max[a] = float(bbox_max[a])
        o.learning_rate = learning_rate
        o.seed = seed
        o.record_capacity = record_capacity
        o.max_depth = max_depth
        h = ctypes.c_void_p()
        N.check(N.lib().rt_guide_create(ctx.handle, ctypes.byref(o), ctypes.byref(h)))
        self.handle = h
        self.opts = o
        self.ctx = ctx  # the context must outlive the guide

    @property
    def param_count(self) -> int:
        n = ctypes.c_uint64()
        N.check(N.lib().rt_guide_param_count(self.handle, ctypes.byref(n)))
        return n.value

    @property
    def steps(self) -> int:
        n = ctypes.c_uint64()
        N.check(N.lib().rt_guide_steps(self.handle, ctypes.byref(n)))
        return n.value

    def reset(self):
        """Seeded initial weights again, Adam state cleared, untrained (device buffers kept)."""
        N.check(N.lib().rt_guide_reset(self.handle))

    def params(self) -> np.ndarray:
        out = np.zeros(self.param_count, dtype=np.float32)
        N.check(N.lib().rt_guide_params_get(self.handle, out.ctypes.data, out.size))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        N.check(N.lib().rt_guide_params_set(self.handle, p.ctypes.data, p.size))

    def eval(self, queries_dev):
        import torch

        B = queries_dev.numel() // 9
        out = torch.empty(B * N.GUIDE_OUTPUTS, dtype=torch.float32, device=queries_dev.device)
        N.check(N.lib().rt_guide_eval(self.handle, queries_dev.data_ptr(), B, out.data_ptr()))
        return out.view(B, N.GUIDE_OUTPUTS)

    def pdf(self, queries_dev, dirs_dev, bsdf_pdf_dev):
        import torch

        B = queries_dev.numel() // 9
        out = torch.empty(B, dtype=torch.float32, device=queries_dev.device)
        N.check(N.lib().rt_guide_pdf(self.handle, queries_dev.data_ptr(), dirs_dev.data_ptr(),
                                     bsdf_pdf_dev.data_ptr(), B, out.data_ptr()))
        return out

    def sample(self, queries_dev, u3_dev):
        import torch

        B = queries_dev.numel() // 9
        dirs = torch.empty(B * 3, dtype=torch.float32, device=queries_dev.device)
        pdf = torch.empty(B, dtype=torch.float32, device=queries_dev.device)
        N.check(N.lib().rt_guide_sample(self.handle, queries_dev.data_ptr(), u3_dev.data_ptr(), B, dirs.data_ptr(),
                                        pdf.data_ptr()))
        return dirs.view(B, 3), pdf

    def train_step(self, queries_dev, dirs_dev, bsdf_pdf_dev, weights_dev, apply: bool = True,
                   want_grad: bool = False):
        """One step; returns (loss, gradient or None)."""
        B = weights_dev.numel()
        grad = np.zeros(self.param_count, dtype=np.float32) if want_grad else None
        loss = ctypes.c_float()
        N.check(N.lib().rt_guide_train_step(self.handle, queries_dev.data_ptr(), dirs_dev.data_ptr(),
                                            bsdf_pdf_dev.data_ptr(), weights_dev.data_ptr(), B, int(apply),
                                            None if grad is None else grad.ctypes.data, ctypes.byref(loss)))
        return loss.value, grad

    def record_count(self):
        r, nz = ctypes.c_uint64(), ctypes.c_uint64()
        N.check(N.lib().rt_guide_record_count(self.handle, ctypes.byref(r), ctypes.byref(nz)))
        return r.value, nz.value

    def records(self) -> np.ndarray:
        """Training records of the last recording render, (n, 20) float32 (see rt_guide_records_get)."""
        n, _ = self.record_count()
        out = np.zeros((n, 20), dtype=np.float32)
        if n:
            N.check(N.lib().rt_guide_records_get(self.handle, 0, n, out.ctypes.data))
        return out

    def train_records(self, steps: int, batch: int = 1 << 18, seed: int = 0) -> float:
        loss = ctypes.c_float()
        N.check(N.lib().rt_guide_train_records(self.handle, steps, batch, seed, ctypes.byref(loss)))
        return loss.value

    def close(self):
        if self.handle:
            N.lib().rt_guide_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def film_store_hdrbmp(path, film, width: int, height: int, samples: int):
    """Film::storeContributionsToFile of a device film: writes `path`.hdrbmp."""
    s64 = film.get("sum64")
    N.check(N.lib().rt_film_store_hdrbmp(str(path).encode(), width, height,
                                         None if s64 is not None else film["sum"].data_ptr(),
                                         film["count"].data_ptr(), None if s64 is None else s64.data_ptr(),
                                         samples))


def film_load_hdrbmp(path, width: int, height: int):
    """Film::loadContributionsFromFile: (per-pixel sums (h*w, 3) float64, samples per pixel)."""
    out = np.zeros((width * height, 3), np.float64)
    n = ctypes.c_uint64()
    N.check(N.lib().rt_film_load_hdrbmp(str(path).encode(), width, height, out.ctypes.data, ctypes.byref(n)))
    return out, n.value


def material_eval(mat, wo, wi):
    """rt_material_eval on (n, 3) host arrays: (f (n, 3), pdf (n,)) as numpy."""
    import torch

    a = torch.from_numpy(np.ascontiguousarray(wo, np.float32).reshape(-1)).cuda()
    b = torch.from_numpy(np.ascontiguousarray(wi, np.float32).reshape(-1)).cuda()
    n = a.numel() // 3
    f = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    pdf = torch.empty(n, dtype=torch.float32, device="cuda")
    N.check(N.lib().rt_material_eval(ctypes.byref(mat), a.data_ptr(), b.data_ptr(), n, f.data_ptr(), pdf.data_ptr()))
    return f.cpu().numpy().reshape(n, 3), pdf.cpu().numpy()


def material_sample(mat, wo, seed: int = 0, flags: int = 0):
    """rt_material_sample on (n, 3) host arrays: (wi, value, pdf, delta) as numpy."""
    import torch

    a = torch.from_numpy(np.ascontiguousarray(wo, np.float32).reshape(-1)).cuda()
    n = a.numel() // 3
    wi = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    val = torch.empty(3 * n, dtype=torch.float32, device="cuda")
    pdf = torch.empty(n, dtype=torch.float32, device="cuda")
    dl = torch.empty(n, dtype=torch.uint8, device="cuda")
    N.check(N.lib().rt_material_sample(ctypes.byref(mat), a.data_ptr(), n, seed, flags, wi.data_ptr(), val.data_ptr(),
                                       pdf.data_ptr(), dl.data_ptr()))
    return (wi.cpu().numpy().reshape(n, 3), val.cpu().numpy().reshape(n, 3), pdf.cpu().numpy(),
            dl.cpu().numpy().astype(bool))


def film_tonemap(film, samples: int, mode: int, use_count: bool = True):
    """Film::toneMaxPixel of a device film (rt_film_tonemap): (H*W, 3) uint8 torch tensor on the
    device, film order. samples: the samples per pixel the film holds."""
    import torch

    npix = film["count"].numel()
    out = torch.empty(npix * 3, dtype=torch.uint8, device="cuda")
    s64 = film.get("sum64")
    N.check(N.lib().rt_film_tonemap(None if s64 is not None else film["sum"].data_ptr(),
                                    film["count"].data_ptr() if use_count else None,
                                    None if s64 is None else s64.data_ptr(), npix, int(samples), mode,
                                    out.data_ptr()))
    return out.view(npix, 3)


def image_write(path, rgb8, width: int, height: int, fmt: str = "bmp"):
    """Writes (H*W, 3) uint8 RGB (host) as the reference's BMP or PPM file."""
    a = np.ascontiguousarray(np.asarray(rgb8, dtype=np.uint8))
    fn = N.lib().rt_image_write_bmp if fmt == "bmp" else N.lib().rt_image_write_ppm
    N.check(fn(str(path).encode(), a.ctypes.data, width, height))


def film_rmse_gpu(film_a, film_b) -> float:
    """computeRMSE of two device films on the GPU (rt_film_rmse)."""
    out = ctypes.c_double()
    a64, b64 = film_a.get("sum64"), film_b.get("sum64")
    N.check(N.lib().rt_film_rmse(None if a64 is not None else film_a["sum"].data_ptr(), film_a["count"].data_ptr(),
                                 None if a64 is None else a64.data_ptr(),
                                 None if b64 is not None else film_b["sum"].data_ptr(), film_b["count"].data_ptr(),
                                 None if b64 is None else b64.data_ptr(), film_a["count"].numel(), ctypes.byref(out)))
    return out.value
