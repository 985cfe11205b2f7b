"""Test infrastructure: ctypes bindings of the two checkers.

* RefOracle: the reference renderer's own code compiled from its sources
  (oracle/_ref/libref_oracle.so, recipe in oracle/Makefile).
* Restated: the plain-C restatement (oracle/_build/librt_oracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's reference/CPU-baseline legs use
these. The product never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_SO = HERE / "_ref" / "libref_oracle.so"
RESTATE_SO = HERE / "_build" / "librt_oracle.so"

P = ctypes.c_void_p
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
I = ctypes.c_int
F = ctypes.c_float


def reference_dir() -> Path | None:
    """The reference source tree named by the REF_DIR environment variable, if it exists."""
    d = os.environ.get("REF_DIR", "")
    return Path(d) if d and Path(d).is_dir() else None


def build(ref: bool = True):
    """Builds the restatement (always) and the reference harnesses when REF_DIR names the
    reference tree. Returns the list of targets built."""
    targets = ["restate"]
    rd = reference_dir()
    if ref and rd is not None:
        targets.append("ref")
    env = dict(os.environ, REF_DIR=str(rd)) if rd is not None else None
    subprocess.run(["make", "-s", "-C", str(HERE), *targets], check=True, env=env)
    return targets


def _np(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class _quiet_stdout:
    """Sends file descriptor 1 to /dev/null for the duration (C code writing to stdout)."""

    def __enter__(self):
        import sys

        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        import ctypes as _c

        _c.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


class RefOracle:
    """The reference's own BVH / triangle / sphere / kd-tree code."""

    def __init__(self, path: Path = REF_SO):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle ref)")
        L = ctypes.CDLL(str(path))
        L.refo_bvh_build.restype = P
        L.refo_bvh_build.argtypes = [P, U32, P, U32, P]
        L.refo_bvh_free.argtypes = [P]
        L.refo_bvh_root.argtypes = [P]
        L.refo_bvh_root.restype = U32
        L.refo_bvh_export.argtypes = [P] * 7
        L.refo_bvh_intersect.argtypes = [P, P, P, P, U64, I, P, I]
        L.refo_bvh_brute.argtypes = [P, P, P, P, U64, I, P, I]
        L.refo_triangle_intersects.argtypes = [P, U32, P, P, F, P, I]
        L.refo_triangle_intersects.restype = I
        L.refo_triangle_hit_t.argtypes = [P, P, P, P, U64, P, I]
        L.refo_spheres_build.restype = P
        L.refo_spheres_build.argtypes = [P, P, P, U32]
        L.refo_spheres_free.argtypes = [P]
        L.refo_sphere_matrices.argtypes = [P, U32, P, P]
        L.refo_spheres_intersect.argtypes = [P, P, P, U64, I, P, P, I]
        L.refo_planes_build.restype = P
        L.refo_planes_build.argtypes = [P, P, U32]
        L.refo_planes_free.argtypes = [P]
        L.refo_plane_matrices.argtypes = [P, U32, P, P]
        L.refo_planes_intersect.argtypes = [P, P, P, U64, I, P, P, I]
        L.refo_kdtree_build.restype = P
        L.refo_kdtree_build.argtypes = [P, P, U64]
        L.refo_kdtree_free.argtypes = [P]
        L.refo_kdtree_knn.argtypes = [P, P, P, U64, U32, F, P, P, I]
        self.L = L

    # ---- BVH
    def bvh(self, verts, idx, transparent=None):
        v = _np(verts, np.float32).reshape(-1, 3)
        i = _np(idx, np.uint32).reshape(-1, 3)
        tr = None if transparent is None else _np(transparent, np.uint8)
        h = self.L.refo_bvh_build(v.ctypes.data, v.shape[0], i.ctypes.data, i.shape[0],
                                  None if tr is None else tr.ctypes.data)
        if not h:
            raise ValueError("reference BVH needs at least 2 triangles")
        return RefBvh(self, h, i.shape[0])


class RefBvh:
    def __init__(self, o: RefOracle, h, ntri):
        self.o, self.h, self.ntri = o, h, ntri

    def __del__(self):
        try:
            self.o.L.refo_bvh_free(self.h)
        except Exception:
            pass

    def export(self):
        nn = 2 * self.ntri - 1
        boxes = np.zeros((nn, 6), np.float32)
        oid = np.zeros(nn, np.int32)
        left = np.zeros(nn, np.uint32)
        right = np.zeros(nn, np.uint32)
        codes = np.zeros(self.ntri, np.uint32)
        srt = np.zeros(self.ntri, np.uint32)
        self.o.L.refo_bvh_export(self.h, boxes.ctypes.data, oid.ctypes.data, left.ctypes.data, right.ctypes.data,
                                 codes.ctypes.data, srt.ctypes.data)
        return dict(boxes=boxes, objectIds=oid, left=left, right=right, codes=codes, sorted=srt,
                    root=self.o.L.refo_bvh_root(self.h))

    def intersect(self, o, d, tmax=None, shadow=False, threads=8, brute=False):
        o = _np(o, np.float32)
        d = _np(d, np.float32)
        tm = None if tmax is None else _np(tmax, np.float32)
        out = np.zeros(o.shape[0], np.int32)
        fn = self.o.L.refo_bvh_brute if brute else self.o.L.refo_bvh_intersect
        fn(self.h, o.ctypes.data, d.ctypes.data, None if tm is None else tm.ctypes.data, o.shape[0], int(shadow),
           out.ctypes.data, threads)
        return out

    def hit_t(self, ids, o, d, threads=8):
        ids = _np(ids, np.int32)
        o = _np(o, np.float32)
        d = _np(d, np.float32)
        t = np.zeros(o.shape[0], np.float32)
        self.o.L.refo_triangle_hit_t(self.h, ids.ctypes.data, o.ctypes.data, d.ctypes.data, o.shape[0],
                                     t.ctypes.data, threads)
        return t

    def triangle_intersects(self, tri, o, d, tmax=np.inf, hit_offset=np.inf, shadow=False):
        o = _np(o, np.float32)
        d = _np(d, np.float32)
        h = np.array([hit_offset], np.float32)
        r = self.o.L.refo_triangle_intersects(self.h, tri, o.ctypes.data, d.ctypes.data, float(tmax), h.ctypes.data,
                                              int(shadow))
        return bool(r), float(h[0])


class RefSpheres:
    def __init__(self, o: RefOracle, centers, radii, glass):
        self.o = o
        c = _np(centers, np.float32).reshape(-1, 3)
        r = _np(radii, np.float32)
        g = _np(glass, np.uint8)
        self.n = c.shape[0]
        self.h = o.L.refo_spheres_build(c.ctypes.data, r.ctypes.data, g.ctypes.data, self.n)

    def __del__(self):
        try:
            self.o.L.refo_spheres_free(self.h)
        except Exception:
            pass

    def matrices(self, i):
        o2w = np.zeros(16, np.float32)
        w2o = np.zeros(16, np.float32)
        self.o.L.refo_sphere_matrices(self.h, i, o2w.ctypes.data, w2o.ctypes.data)
        return o2w.reshape(4, 4), w2o.reshape(4, 4)

    def intersect(self, o, d, shadow=False, threads=8):
        o = _np(o, np.float32)
        d = _np(d, np.float32)
        ids = np.zeros(o.shape[0], np.int32)
        t = np.zeros(o.shape[0], np.float32)
        self.o.L.refo_spheres_intersect(self.h, o.ctypes.data, d.ctypes.data, o.shape[0], int(shadow), ids.ctypes.data,
                                        t.ctypes.data, threads)
        return ids, t


class RefPlanes:
    """The reference's Plane shapes (Plane(bottomLeftCorner, axisX, axisY, normal)), their
    matrices and Plane::intersects in Scene::intersects' shape-loop order."""

    def __init__(self, o: RefOracle, planes12, glass=None):
        self.o = o
        p = _np(planes12, np.float32).reshape(-1, 12)
        g = None if glass is None else _np(glass, np.uint8)
        self.n = p.shape[0]
        self.h = o.L.refo_planes_build(p.ctypes.data, None if g is None else g.ctypes.data, self.n)

    def __del__(self):
        if getattr(self, "h", None):
            self.o.L.refo_planes_free(self.h)
            self.h = None

    def matrices(self, i):
        o2w, w2o = np.zeros(16, np.float32), np.zeros(16, np.float32)
        self.o.L.refo_plane_matrices(self.h, i, o2w.ctypes.data, w2o.ctypes.data)
        return o2w.reshape(4, 4), w2o.reshape(4, 4)

    def intersect(self, o, d, t_init=None, shadow=False, threads=8):
        """(ids, t): the last plane that lowered the running offset (starting at t_init), -1: none."""
        o = _np(o, np.float32).reshape(-1, 3)
        d = _np(d, np.float32).reshape(-1, 3)
        n = o.shape[0]
        t = np.full(n, np.inf, np.float32) if t_init is None else _np(t_init, np.float32).copy()
        ids = np.zeros(n, np.int32)
        self.o.L.refo_planes_intersect(self.h, o.ctypes.data, d.ctypes.data, n, int(shadow), ids.ctypes.data,
                                       t.ctypes.data, threads)
        return ids, t


class RefKdTree:
    def __init__(self, o: RefOracle, pos, shape_ids=None):
        self.o = o
        p = _np(pos, np.float32).reshape(-1, 3)
        s = None if shape_ids is None else _np(shape_ids, np.int32)
        self.h = o.L.refo_kdtree_build(p.ctypes.data, None if s is None else s.ctypes.data, p.shape[0])

    def __del__(self):
        try:
            self.o.L.refo_kdtree_free(self.h)
        except Exception:
            pass

    def knn(self, q, k, radius, qshape=None, threads=8):
        q = _np(q, np.float32).reshape(-1, 3)
        qs = None if qshape is None else _np(qshape, np.int32)
        idx = np.zeros((q.shape[0], k), np.int32)
        cnt = np.zeros(q.shape[0], np.uint32)
        self.o.L.refo_kdtree_knn(self.h, q.ctypes.data, None if qs is None else qs.ctypes.data, q.shape[0], k,
                                 float(radius), idx.ctypes.data, cnt.ctypes.data, threads)
        return idx, cnt


class Restated:
    """The C restatement (oracle/rt_oracle.c)."""

    def __init__(self, path: Path = RESTATE_SO):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle restate)")
        L = ctypes.CDLL(str(path))
        L.rto_bvh_build.argtypes = [P, U32, P, U32, P, ctypes.POINTER(P)]
        L.rto_bvh_build.restype = I
        L.rto_bvh_free.argtypes = [P]
        L.rto_bvh_export.argtypes = [P, P, P, P]
        L.rto_bvh_tie_rank.argtypes = [P, P]
        L.rto_trace_ref_order.argtypes = [P, P, P, P, U64, I, P, P, I]
        L.rto_triangle_intersects.argtypes = [P, U32, P, P, F, P, I]
        L.rto_triangle_intersects.restype = I
        L.rto_sphere_intersects.argtypes = [P, F, P, P, F, P]
        L.rto_sphere_intersects.restype = I
        L.rto_knn_brute.argtypes = [P, P, U64, P, P, U64, U32, F, P, P, P, I]
        self.L = L

    def bvh(self, verts, idx, transparent=None):
        v = _np(verts, np.float32).reshape(-1, 3)
        i = _np(idx, np.uint32).reshape(-1, 3)
        tr = None if transparent is None else _np(transparent, np.uint8)
        h = P()
        if self.L.rto_bvh_build(v.ctypes.data, v.shape[0], i.ctypes.data, i.shape[0],
                                None if tr is None else tr.ctypes.data, ctypes.byref(h)) != 0:
            raise ValueError("rto_bvh_build failed")
        return RestatedBvh(self, h, i.shape[0])

    def sphere_intersects(self, w2o, radius, o, d, tmax=np.inf, hit_offset=np.inf):
        m = _np(w2o, np.float32).reshape(16)
        o = _np(o, np.float32)
        d = _np(d, np.float32)
        h = np.array([hit_offset], np.float32)
        r = self.L.rto_sphere_intersects(m.ctypes.data, float(radius), o.ctypes.data, d.ctypes.data, float(tmax),
                                         h.ctypes.data)
        return bool(r), float(h[0])

    def knn(self, pos, shape, q, qshape, k, radius, threads=8):
        p = _np(pos, np.float32).reshape(-1, 3)
        s = _np(shape, np.int32)
        q = _np(q, np.float32).reshape(-1, 3)
        qs = None if qshape is None else _np(qshape, np.int32)
        idx = np.zeros((q.shape[0], k), np.int32)
        dist = np.zeros((q.shape[0], k), np.float32)
        cnt = np.zeros(q.shape[0], np.uint32)
        self.L.rto_knn_brute(p.ctypes.data, s.ctypes.data, p.shape[0], q.ctypes.data,
                             None if qs is None else qs.ctypes.data, q.shape[0], k, float(radius), idx.ctypes.data,
                             dist.ctypes.data, cnt.ctypes.data, threads)
        return idx, dist, cnt


def restated_phong_eval(restated, material, wo, wi):
    """The CPU restatement's Phong BSDF (f * |cos|, pdf) for pairs of shading-space directions."""
    import importlib

    N = importlib.import_module("2023_render_engine_b200._native")
    L = restated.L
    L.pto_phong_eval.argtypes = [ctypes.POINTER(N.Material), P, P, U32, P, P]
    a, b = _np(wo, np.float32).reshape(-1, 3), _np(wi, np.float32).reshape(-1, 3)
    f = np.zeros((a.shape[0], 3), np.float32)
    pdf = np.zeros(a.shape[0], np.float32)
    L.pto_phong_eval(ctypes.byref(material), a.ctypes.data, b.ctypes.data, a.shape[0], f.ctypes.data, pdf.ctypes.data)
    return f, pdf


def ref_material_eval(refo, kind, kd, eta, k, rx, ry, wo, wi):
    """Material::lightReflected / pdf of the reference's own class (kind: rt_material_type)."""
    L = refo.L
    L.refo_material_eval.argtypes = [I, P, P, P, ctypes.c_float, ctypes.c_float, P, P, U32, P, P]
    L.refo_material_eval.restype = I
    a, b = _np(wo, np.float32).reshape(-1, 3), _np(wi, np.float32).reshape(-1, 3)
    p = [_np(x, np.float32) for x in (kd, eta, k)]
    f = np.zeros((a.shape[0], 3), np.float32)
    pdf = np.zeros(a.shape[0], np.float32)
    if L.refo_material_eval(kind, *[x.ctypes.data for x in p], rx, ry, a.ctypes.data, b.ctypes.data, a.shape[0],
                            f.ctypes.data, pdf.ctypes.data) != 0:
        raise ValueError(f"unknown material kind {kind}")
    return f, pdf


def write_bmp24(path, rgb_rows):
    """A 24-bit BMP as Texture::loadBmpImage (textures/Texture.cu:38-121) reads it: `rgb_rows`
    (height, width, 3) uint8, row i = the i-th row stored in the file, BGR on disk. The width
    must make a row a multiple of 4 bytes (the reader does not skip row padding)."""
    a = np.ascontiguousarray(rgb_rows, dtype=np.uint8)
    h, w, _ = a.shape
    if (3 * w) % 4:
        raise ValueError("row bytes must be a multiple of 4")
    import struct

    data = a[:, :, ::-1].tobytes()
    hdr = struct.pack("<2sIHHIIiiHHIIiiII", b"BM", 54 + len(data), 0, 0, 54, 40, w, h, 1, 24, 0, len(data), 2835, 2835,
                      0, 0)
    Path(path).write_bytes(hdr + data)


def ref_texture_lookup(refo, bmp_path, uv):
    """Texture::getColor of the reference's own Texture read from bmp_path."""
    L = refo.L
    L.refo_texture_lookup.argtypes = [ctypes.c_char_p, P, U32, P]
    L.refo_texture_lookup.restype = I
    u = _np(uv, np.float32).reshape(-1, 2)
    out = np.zeros((u.shape[0], 3), np.float32)
    if L.refo_texture_lookup(str(bmp_path).encode(), u.ctypes.data, u.shape[0], out.ctypes.data) != 0:
        raise FileNotFoundError(bmp_path)
    return out


def ref_material_eval_tex(refo, kind, kd, eta, k, rx, ry, bmp_path, uv, wo, wi):
    """lightReflected / pdf of the reference's class with a Texture, pair i at surface point uv[i]
    (kind: 0 Lambertian, 1 Trowbridge, 5 Phong with ks = eta and ns = rx, 8 Beckmann, 9
    TrowbridgeBasic)."""
    L = refo.L
    L.refo_material_eval_tex.argtypes = [I, P, P, P, ctypes.c_float, ctypes.c_float, ctypes.c_char_p, P, P, P, U32,
                                         P, P]
    L.refo_material_eval_tex.restype = I
    a, b = _np(wo, np.float32).reshape(-1, 3), _np(wi, np.float32).reshape(-1, 3)
    u = _np(uv, np.float32).reshape(-1, 2)
    p = [_np(x, np.float32) for x in (kd, eta, k)]
    f = np.zeros((a.shape[0], 3), np.float32)
    pdf = np.zeros(a.shape[0], np.float32)
    rc = L.refo_material_eval_tex(kind, *[x.ctypes.data for x in p], rx, ry, str(bmp_path).encode(), u.ctypes.data,
                                  a.ctypes.data, b.ctypes.data, a.shape[0], f.ctypes.data, pdf.ctypes.data)
    if rc != 0:
        raise ValueError(f"reference textured material eval failed ({rc})")
    return f, pdf


def ref_phong_eval(refo, kd, ks, ns, wo, wi):
    """The reference's PhongMaterial::lightReflected / pdf."""
    L = refo.L
    L.refo_phong_eval.argtypes = [P, P, ctypes.c_float, P, P, U32, P, P]
    a, b = _np(wo, np.float32).reshape(-1, 3), _np(wi, np.float32).reshape(-1, 3)
    kd_, ks_ = _np(kd, np.float32), _np(ks, np.float32)
    f = np.zeros((a.shape[0], 3), np.float32)
    pdf = np.zeros(a.shape[0], np.float32)
    L.refo_phong_eval(kd_.ctypes.data, ks_.ctypes.data, ns, a.ctypes.data, b.ctypes.data, a.shape[0], f.ctypes.data,
                      pdf.ctypes.data)
    return f, pdf


def ref_diffusion_term(refo, cam_p, cam_dir, cam_n, ph_loc, ph_dir, ph_n, sigma_s, sigma_a, g, eta):
    """The reference's diffusionTermBSSRDF (geometricMath.cu:500-522) for one photon (rgb)."""
    L = refo.L
    L.refo_diffusion_term.argtypes = [P, P, P, P, P, P, P, P, ctypes.c_float, ctypes.c_float, P]
    args = [_np(x, np.float32) for x in (cam_p, cam_dir, cam_n, ph_loc, ph_dir, ph_n, sigma_s, sigma_a)]
    out = np.zeros(3, np.float64)
    L.refo_diffusion_term(*[a.ctypes.data for a in args], g, eta, out.ctypes.data)
    return out


class RestatedBvh:
    def __init__(self, o: Restated, h, ntri):
        self.o, self.h, self.ntri = o, h, ntri

    def __del__(self):
        try:
            self.o.L.rto_bvh_free(self.h)
        except Exception:
            pass

    def export(self):
        boxes = np.zeros((2 * self.ntri - 1, 6), np.float32)
        codes = np.zeros(self.ntri, np.uint32)
        srt = np.zeros(self.ntri, np.uint32)
        self.o.L.rto_bvh_export(self.h, boxes.ctypes.data, codes.ctypes.data, srt.ctypes.data)
        return dict(boxes=boxes, codes=codes, sorted=srt)

    def tie_rank(self):
        r = np.zeros(self.ntri, np.uint32)
        self.o.L.rto_bvh_tie_rank(self.h, r.ctypes.data)
        return r

    def intersect(self, o, d, tmax=None, shadow=False, threads=8):
        o = _np(o, np.float32)
        d = _np(d, np.float32)
        tm = None if tmax is None else _np(tmax, np.float32)
        out = np.zeros(o.shape[0], np.int32)
        t = np.zeros(o.shape[0], np.float32)
        self.o.L.rto_trace_ref_order(self.h, o.ctypes.data, d.ctypes.data, None if tm is None else tm.ctypes.data,
                                     o.shape[0], int(shadow), out.ctypes.data, t.ctypes.data, threads)
        return out, t

    def triangle_intersects(self, tri, o, d, tmax=np.inf, hit_offset=np.inf, shadow=False):
        o = _np(o, np.float32)
        d = _np(d, np.float32)
        h = np.array([hit_offset], np.float32)
        r = self.o.L.rto_triangle_intersects(self.h, tri, o.ctypes.data, d.ctypes.data, float(tmax), h.ctypes.data,
                                             int(shadow))
        return bool(r), float(h[0])


class PathTracerOracle:
    """CPU restatement of the renderer's estimator (oracle/pt_oracle.c) over a scene
    given as a triangle soup + spheres + materials + point lights."""

    def __init__(self, restated: Restated, verts, idx, tri_mat, spheres, materials, plights=()):
        import importlib

        N = importlib.import_module("2023_render_engine_b200._native")
        L = restated.L
        L.pto_render.argtypes = [P, P, P, U32, P, U32, P, U32, P, U32, U32, U32, U32, U32, U32, U32, U32, P, P, I]
        L.pto_render.restype = I
        self.L = L
        self.bvh = restated.bvh(verts, idx) if len(idx) else None
        self.tri_mat = _np(tri_mat, np.uint32)
        sph = np.zeros(len(spheres), dtype=np.dtype([("w2o", "<f4", 16), ("o2w", "<f4", 16), ("radius", "<f4"),
                                                      ("material", "<u4")]))
        for i, s in enumerate(spheres):
            sph[i]["w2o"] = np.asarray(s["w2o"], np.float32).reshape(16)
            sph[i]["o2w"] = np.asarray(s["o2w"], np.float32).reshape(16)
            sph[i]["radius"] = s["radius"]
            sph[i]["material"] = s["material"]
        self.sph = sph
        self.mats = (N.Material * len(materials))(*materials)
        self.nmat = len(materials)
        self.pl = _np(np.array([list(p) + list(np.asarray(c) * i) for p, c, i in plights], np.float32).reshape(-1),
                      np.float32) if len(plights) else np.zeros(6, np.float32)
        self.npl = len(plights)

    def render(self, camera, spp, max_depth, rr_depth=3, seed=0, flags=0, sample_offset=0, threads=8,
               pixels=None):
        w, h = camera.width, camera.height
        p0, p1 = (0, w * h) if pixels is None else pixels
        s = np.zeros((w * h, 3), np.float64)
        c = np.zeros(w * h, np.uint32)
        self.L.pto_render(self.bvh.h if self.bvh is not None else None, self.tri_mat.ctypes.data,
                          self.sph.ctypes.data if len(self.sph) else None, len(self.sph),
                          ctypes.cast(self.mats, ctypes.c_void_p), self.nmat, self.pl.ctypes.data, self.npl,
                          ctypes.addressof(camera), spp, sample_offset, max_depth, rr_depth, seed, flags, p0, p1,
                          s.ctypes.data, c.ctypes.data, threads)
        return s, c

    def trace_photons(self, tri_shape, sph_shape, plights, n, max_depth=30, rr_depth=3, seed=0, flags=0, cap=None):
        """plights: list of (pos, rgb, intensity). Returns photons as a structured array."""
        import importlib

        N = importlib.import_module("2023_render_engine_b200._native")
        L = self.L
        L.pto_trace_photons.argtypes = [P, P, P, P, P, U32, P, U32, P, P, U32, U64, U32, U32, U32, U32, P, U64]
        L.pto_trace_photons.restype = U64
        pl = np.array([list(p) + list(np.asarray(c, np.float64) * i) for p, c, i in plights], np.float32)
        rgbi = np.array([list(c) + [i] for p, c, i in plights], np.float32)
        ts = _np(tri_shape, np.int32)
        ss = _np(sph_shape, np.int32) if len(sph_shape) else np.zeros(1, np.int32)
        cap = cap or 8 * n
        out = np.zeros(cap, dtype=N.PHOTON_DTYPE)
        got = L.pto_trace_photons(self.bvh.h if self.bvh is not None else None, self.tri_mat.ctypes.data,
                                  ts.ctypes.data, self.sph.ctypes.data if len(self.sph) else None, ss.ctypes.data,
                                  len(self.sph), ctypes.cast(self.mats, ctypes.c_void_p), self.nmat, pl.ctypes.data,
                                  rgbi.ctypes.data, len(plights), n, max_depth, rr_depth, seed, flags,
                                  out.ctypes.data, cap)
        return out[:min(got, cap)]


class RefRender:
    """The reference's own PathTracerIntegrator on a plane + point-light scene
    (oracle/_ref/libref_render.so; image size, spp and depth fixed at its compile time)."""

    def __init__(self, path=HERE / "_ref" / "libref_render.so"):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle ref)")
        L = ctypes.CDLL(str(path))
        L.refr_config.argtypes = [P, P, P, P]
        L.refr_render.argtypes = [ctypes.c_char_p, I, P, P, P, P, P]
        L.refr_render.restype = I
        self.L = L
        w, h, s, d = (ctypes.c_int() for _ in range(4))
        L.refr_config(ctypes.byref(w), ctypes.byref(h), ctypes.byref(s), ctypes.byref(d))
        self.width, self.height, self.spp, self.depth = w.value, h.value, s.value, d.value

    def single_scattering(self, eta, ns, g, sigma_s, sigma_a, wo, L, seeds):
        """SSMaterial::singleScattering of the reference's class: (value (n, 3), Ti (n, 3),
        Pi (n, 3), the sample u each case drew (n,))."""
        L_ = self.L
        L_.refr_single_scattering.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float, P, P, P, P, P, U32, P,
                                              P, P, P]
        L_.refr_single_scattering.restype = I
        a, b = _np(wo, np.float32).reshape(-1, 3), _np(L, np.float32).reshape(-1, 3)
        sd = _np(seeds, np.uint32)
        ss, sa = _np(sigma_s, np.float32), _np(sigma_a, np.float32)
        n = a.shape[0]
        v, wi, pt, u = (np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32),
                        np.zeros(n, np.float32))
        L_.refr_single_scattering(eta, ns, g, ss.ctypes.data, sa.ctypes.data, a.ctypes.data, b.ctypes.data,
                                  sd.ctypes.data, n, v.ctypes.data, wi.ctypes.data, pt.ctypes.data, u.ctypes.data)
        return v, wi, pt, u

    def film_store(self, path, sums, samples):
        """Film::storeContributionsToFile of a film with these per-pixel sums (h*w, 3)."""
        a = _np(sums, np.float64).reshape(-1, 3)
        L = self.L
        L.refr_film_store.argtypes = [ctypes.c_char_p, P, ctypes.c_longlong]
        L.refr_film_store(str(path).encode(), a.ctypes.data, samples)

    def film_load(self, path):
        """Film::loadContributionsFromFile: (sums (h*w, 3), samples)."""
        L = self.L
        L.refr_film_load.argtypes = [ctypes.c_char_p, P, P]
        out = np.zeros((self.width * self.height, 3), np.float64)
        n = ctypes.c_longlong()
        if L.refr_film_load(str(path).encode(), out.ctypes.data, ctypes.byref(n)) != 0:
            raise RuntimeError("reference film load failed")
        return out, n.value

    def film_write(self, path, sums, samples, mode, bmp=True):
        """Film::writeToBMP / writeToPPM of a film with these sums: writes path + '.bmp' / '.ppm'."""
        a = _np(sums, np.float64).reshape(-1, 3)
        L = self.L
        L.refr_film_write.argtypes = [ctypes.c_char_p, P, ctypes.c_longlong, I, I]
        L.refr_film_write(str(path).encode(), a.ctypes.data, samples, mode, int(bmp))

    def bmp_write(self, path, bgr_rows, width, height):
        """BitmapImage::write_image of (height, width, 3) BGR bytes, file row order (bottom-up)."""
        a = np.ascontiguousarray(bgr_rows, np.uint8)
        L = self.L
        L.refr_bmp_write.argtypes = [ctypes.c_char_p, P, I, I]
        L.refr_bmp_write(str(path).encode(), a.ctypes.data, width, height)

    def film_rmse(self, a, na, b, nb):
        """computeRMSE of two films given by per-pixel sums and samples per pixel."""
        L = self.L
        L.refr_film_rmse.argtypes = [P, ctypes.c_longlong, P, ctypes.c_longlong]
        L.refr_film_rmse.restype = ctypes.c_double
        a = _np(a, np.float64).reshape(-1, 3)
        b = _np(b, np.float64).reshape(-1, 3)
        return L.refr_film_rmse(a.ctypes.data, na, b.ctypes.data, nb)

    def render(self, obejota_path, planes, kd, bmp_path=None, textured=None):
        """planes: (n, 12) Plane(corner, axisX, axisY, normal); kd: (n, 3); textured: per plane
        whether its material carries the Texture read from bmp_path. Returns (mean image
        (h*w, 3), cameraToWorld 4x4, rasterToCamera 4x4)."""
        pl = _np(planes, np.float32).reshape(-1, 12)
        k = _np(kd, np.float32).reshape(-1, 3)
        out = np.zeros((self.width * self.height, 3), np.float32)
        c2w = np.zeros(16, np.float32)
        r2c = np.zeros(16, np.float32)
        L = self.L
        L.refr_render_tex.argtypes = [ctypes.c_char_p, I, P, P, ctypes.c_char_p, P, P, P, P]
        L.refr_render_tex.restype = I
        tx = None if textured is None else _np(textured, np.int32)
        rc = L.refr_render_tex(str(obejota_path).encode(), pl.shape[0], pl.ctypes.data, k.ctypes.data,
                               None if bmp_path is None else str(bmp_path).encode(),
                               None if tx is None else tx.ctypes.data, out.ctypes.data, c2w.ctypes.data,
                               r2c.ctypes.data)
        if rc != 0:
            raise RuntimeError("reference render failed")
        return out, c2w.reshape(4, 4), r2c.reshape(4, 4)


class RefCompat:
    """The reference's own scene objects (Plane shapes, Lambertian materials, its .obejota
    camera and point lights) rendered by this repository's core through
    include/rt_b200_compat.hpp (oracle/_ref/libref_compat.so)."""

    def __init__(self, path=HERE / "_ref" / "libref_compat.so"):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle ref)")
        L = ctypes.CDLL(str(path))
        L.refc_config.argtypes = [P, P, P, P]
        L.refc_render.argtypes = [ctypes.c_char_p, I, P, P, ctypes.c_uint32, P]
        L.refc_render.restype = I
        L.refc_error.restype = ctypes.c_char_p
        L.refc_map_material.argtypes = [I, P, P, P, ctypes.c_float, ctypes.c_float, P]
        L.refc_map_material.restype = I
        self.L = L
        w, h, s, d = (ctypes.c_int() for _ in range(4))
        L.refc_config(ctypes.byref(w), ctypes.byref(h), ctypes.byref(s), ctypes.byref(d))
        self.width, self.height, self.spp, self.depth = w.value, h.value, s.value, d.value

    def render(self, obejota_path, planes, kd, seed, bmp_path=None, textured=None):
        pl = _np(planes, np.float32).reshape(-1, 12)
        k = _np(kd, np.float32).reshape(-1, 3)
        out = np.zeros((self.width * self.height, 3), np.float32)
        L = self.L
        L.refc_render_tex.argtypes = [ctypes.c_char_p, I, P, P, ctypes.c_char_p, P, U32, P]
        L.refc_render_tex.restype = I
        tx = None if textured is None else _np(textured, np.int32)
        rc = L.refc_render_tex(str(obejota_path).encode(), pl.shape[0], pl.ctypes.data, k.ctypes.data,
                               None if bmp_path is None else str(bmp_path).encode(),
                               None if tx is None else tx.ctypes.data, seed, out.ctypes.data)
        if rc != 0:
            raise RuntimeError("compat render failed: " + self.L.refc_error().decode())
        return out


class RefCuda:
    """The reference's own GPU traversal (BVH::intersectRay via thrust::transform) built with
    the flags of its compile.sh (oracle/_ref/libref_cuda.so): the reference-CUDA baseline."""

    def __init__(self, path=HERE / "_ref" / "libref_cuda.so"):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle ref)")
        L = ctypes.CDLL(str(path))
        L.refg_build.argtypes = [P, ctypes.c_uint32, P, ctypes.c_uint32]
        L.refg_build.restype = P
        L.refg_free.argtypes = [P]
        L.refg_trace.argtypes = [P, P, ctypes.c_uint64, ctypes.c_int32, P, P, P]
        L.refg_trace.restype = I
        L.refg_error.restype = ctypes.c_char_p
        self.L = L

    def build(self, verts, idx):
        v = _np(verts, np.float32).reshape(-1, 3)
        f = _np(idx, np.uint32).reshape(-1, 3)
        h = self.L.refg_build(v.ctypes.data, v.shape[0], f.ctypes.data, f.shape[0])
        if not h:
            raise RuntimeError("reference GPU BVH build failed: " + self.L.refg_error().decode())
        return h

    def free(self, h):
        self.L.refg_free(h)

    def trace(self, h, o, d, reps=3):
        """Returns (ids, ms per transform with device-resident rays, ms per API-style call)."""
        od = np.ascontiguousarray(np.concatenate([_np(o, np.float32).reshape(-1, 3), _np(d, np.float32).reshape(-1, 3)],
                                                 axis=1))
        n = od.shape[0]
        ids = np.zeros(n, np.int32)
        mk, ma = ctypes.c_float(), ctypes.c_float()
        rc = self.L.refg_trace(h, od.ctypes.data, n, reps, ids.ctypes.data, ctypes.byref(mk), ctypes.byref(ma))
        if rc != 0:
            raise RuntimeError("reference GPU trace failed: " + self.L.refg_error().decode())
        return ids, mk.value, ma.value


class RefIntegrator:
    """The reference's own PathTracerIntegrator::render (with Scene::build and its BVH) on
    triangle meshes, spheres and planes (oracle/ref_integrator_harness.cu).

    host=True: libref_integrator_host.so, the host-compiled integrator (thrust's device system
    on OpenMP: its BVH build and traversal run on the host cores too). host=False:
    libref_integrator_cuda.so, its stock CUDA build (BVH on the GPU, compile.sh flags)."""

    # material kinds of the harness's 16-float table entries
    LAMBERTIAN, TROWBRIDGE, LIGHT, DIELECTRIC, MIRROR, SUBSURFACE = 0, 1, 2, 3, 4, 5
    PATH_TRACING, PHOTON_MAPPING, HYBRID = 0, 1, 2

    def __init__(self, host: bool = True):
        name = "libref_integrator_host.so" if host else "libref_integrator_cuda.so"
        path = HERE / "_ref" / name
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle ref)")
        L = ctypes.CDLL(str(path))
        L.refi_error.restype = ctypes.c_char_p
        L.refi_config.argtypes = [I, I, I, I]
        L.refi_config_photons.argtypes = [I, I, U32, U32, F]
        L.refi_config_photons.restype = I
        L.refi_render.argtypes = [ctypes.c_char_p, U32, P, U32, P, P, P, U32, P, P, U32, P, P, U32, P, P, P, P, P]
        L.refi_render.restype = I
        L.refi_material_sample.argtypes = [P, P, P, U32, P, P, P]
        L.refi_material_sample.restype = I
        L.refi_photons.argtypes = [ctypes.c_char_p, U32, P, U32, P, P, P, U32, P, P, U32, P, P, U32, P, U32, P, P, P,
                                   U64, P]
        L.refi_photons.restype = I
        self.L = L
        self.host = bool(L.refi_host_backend())

    @staticmethod
    def entry(kind, color=(1, 1, 1), eta=(0, 0, 0), k=(0, 0, 0), roughness=(0, 0), value=0.0):
        """A material table entry: value is the Light intensity or the Dielectric IOR."""
        e = np.zeros(16, np.float32)
        e[0] = kind
        e[1:4] = color
        if kind == RefIntegrator.TROWBRIDGE:
            e[4:7], e[7:10], e[10:12] = eta, k, roughness
        else:
            e[4] = value
        return e

    @staticmethod
    def subsurface_entry(kd, ks, eta, ns, sigma_s, sigma_a, g):
        """SSMaterial(0, kd, ks, eta, ns, no texture, opaque, sigma_s, sigma_a, g)."""
        e = np.zeros(16, np.float32)
        e[0] = RefIntegrator.SUBSURFACE
        e[1:4], e[4:7], e[7], e[8] = kd, ks, eta, ns
        e[9:12], e[12:15], e[15] = sigma_s, sigma_a, g
        return e

    def config_photons(self, mode, subsurface, photons, neighbours, radius):
        """RENDER_MODE, CHECK_SUBSURFACE_SCATTERING, N_PHOTON_SAMPLES, MAX_NEIGHBOURS and
        PHOTON_SEARCH_RADIUS of the reference's render (types.h:51-60)."""
        if self.L.refi_config_photons(int(mode), int(bool(subsurface)), int(photons), int(neighbours),
                                      float(radius)) != 0:
            raise ValueError("bad photon configuration")

    def render(self, obejota_path, width, height, spp, depth, materials, verts=None, idx=None, tri_mat=None,
               tri_shape=None, spheres=(), planes=()):
        """Returns (per-pixel mean (h*w, 3), camera_to_world (4, 4), raster_to_camera (4, 4), stats)
        with stats = {render_s, extension_rays, shadow_rays, build_s}. spheres: (center, radius,
        material); planes: (12 floats of Plane(corner, axisX, axisY, normal), material)."""
        if self.L.refi_config(width, height, spp, depth) != 0:
            raise ValueError("bad render configuration")
        mats = _np(np.stack(list(materials)), np.float32).reshape(-1, 16)
        if verts is None or idx is None or len(idx) == 0:
            v = np.zeros((1, 3), np.float32)
            f = np.zeros((0, 3), np.uint32)
        else:
            v, f = _np(verts, np.float32).reshape(-1, 3), _np(idx, np.uint32).reshape(-1, 3)
        tm = _np(tri_mat if tri_mat is not None else np.zeros(f.shape[0]), np.uint32)
        ts = _np(tri_shape if tri_shape is not None else np.zeros(f.shape[0]), np.int32)
        sp = _np([[*c, r] for c, r, _ in spheres], np.float32).reshape(-1, 4)
        spm = _np([m for _, _, m in spheres], np.uint32)
        pl = _np([p for p, _ in planes], np.float32).reshape(-1, 12)
        plm = _np([m for _, m in planes], np.uint32)
        out = np.zeros((width * height, 3), np.float32)
        c2w, r2c, st = np.zeros(16, np.float32), np.zeros(16, np.float32), np.zeros(4, np.float64)
        with _quiet_stdout():  # the integrator printf()s progress lines
            rc = self.L.refi_render(str(obejota_path).encode(), v.shape[0], v.ctypes.data, f.shape[0], f.ctypes.data,
                                    tm.ctypes.data, ts.ctypes.data, sp.shape[0], sp.ctypes.data, spm.ctypes.data,
                                    pl.shape[0], pl.ctypes.data, plm.ctypes.data, mats.shape[0], mats.ctypes.data,
                                    out.ctypes.data, c2w.ctypes.data, r2c.ctypes.data, st.ctypes.data)
        if rc != 0:
            raise RuntimeError("reference render failed: " + self.L.refi_error().decode())
        stats = dict(render_s=float(st[0]), extension_rays=int(st[1]), shadow_rays=int(st[2]), build_s=float(st[3]))
        return out, c2w.reshape(4, 4), r2c.reshape(4, 4), stats

    @staticmethod
    def _scene_args(materials, verts, idx, tri_mat, tri_shape, spheres, planes):
        mats = _np(np.stack(list(materials)), np.float32).reshape(-1, 16)
        if verts is None or idx is None or len(idx) == 0:
            v, f = np.zeros((1, 3), np.float32), np.zeros((0, 3), np.uint32)
        else:
            v, f = _np(verts, np.float32).reshape(-1, 3), _np(idx, np.uint32).reshape(-1, 3)
        tm = _np(tri_mat if tri_mat is not None else np.zeros(f.shape[0]), np.uint32)
        ts = _np(tri_shape if tri_shape is not None else np.zeros(f.shape[0]), np.int32)
        sp = _np([[*c, r] for c, r, _ in spheres], np.float32).reshape(-1, 4)
        spm = _np([m for _, _, m in spheres], np.uint32)
        pl = _np([p for p, _ in planes], np.float32).reshape(-1, 12)
        plm = _np([m for _, m in planes], np.uint32)
        keep = (mats, v, f, tm, ts, sp, spm, pl, plm)
        args = [v.shape[0], v.ctypes.data, f.shape[0], f.ctypes.data, tm.ctypes.data, ts.ctypes.data, sp.shape[0],
                sp.ctypes.data, spm.ctypes.data, pl.shape[0], pl.ctypes.data, plm.ctypes.data, mats.shape[0],
                mats.ctypes.data]
        return keep, args

    def photons(self, obejota_path, nphotons, materials, verts=None, idx=None, tri_mat=None, tri_shape=None,
                spheres=(), planes=(), cap=None):
        """The reference's photon pass (generatePhotons) with nphotons emitted: the stored photons
        as (positions (n, 3), power (n, 3), shape ids (n,))."""
        keep, args = self._scene_args(materials, verts, idx, tri_mat, tri_shape, spheres, planes)
        cap = cap or 8 * nphotons
        pos, power = np.zeros((cap, 3), np.float32), np.zeros((cap, 3), np.float32)
        shape = np.zeros(cap, np.int32)
        count = ctypes.c_uint64()
        with _quiet_stdout():
            rc = self.L.refi_photons(str(obejota_path).encode(), *args, nphotons, pos.ctypes.data, power.ctypes.data,
                                     shape.ctypes.data, cap, ctypes.byref(count))
        del keep
        if rc != 0:
            raise RuntimeError("reference photon pass failed: " + self.L.refi_error().decode())
        n = min(count.value, cap)
        return pos[:n], power[:n], shape[:n]

    def material_sample(self, entry, wo, seeds):
        """Material::sampleDirection of the reference's class: (wi (n, 3), value (n, 3), the
        first 1D sample each case drew (n,))."""
        a = _np(wo, np.float32).reshape(-1, 3)
        sd = _np(seeds, np.uint32)
        n = a.shape[0]
        wi, val, u = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        e = _np(entry, np.float32)
        if self.L.refi_material_sample(e.ctypes.data, a.ctypes.data, sd.ctypes.data, n, wi.ctypes.data,
                                       val.ctypes.data, u.ctypes.data) != 0:
            raise RuntimeError(self.L.refi_error().decode())
        return wi, val, u
