"""Closest-hit parity of the CUDA path (through the C ABI) with the reference's own
traversal: bit-exact triangle ids and hit distances."""
import hashlib
import importlib
import json

import numpy as np
import pytest

import cases
from conftest import GOLDEN

S = importlib.import_module("2023_render_engine_b200.scenes")
N = importlib.import_module("2023_render_engine_b200._native")

pytestmark = pytest.mark.gpu


def _unpack(z, key):
    return {k.split("__", 1)[1]: z[k] for k in z.files if k.startswith(key + "__")}


def make_scene(core, ctx, v, f, transparent=None, spheres=()):
    sc = core.Scene(ctx)
    if f.shape[0]:
        if transparent is None:
            sc.add_mesh(v, f)
        else:  # one mesh per triangle run with equal transparency, keeping global order
            tr = np.asarray(transparent).astype(bool)
            start = 0
            while start < len(tr):
                end = start
                while end < len(tr) and tr[end] == tr[start]:
                    end += 1
                sc.add_mesh(v, f[start:end], transparent=bool(tr[start]))
                start = end
    for s in spheres:
        sc.add_sphere(s["o2w"], s["w2o"], s["radius"], transparent=s.get("glass", False))
    sc.commit()
    return sc


def trace_gpu(sc, o, d, tmax=None, flags=0):
    import torch

    rays = core_make_rays(o, d, tmax)
    rd = torch.from_numpy(rays.view(np.float32).reshape(-1)).cuda()
    hd = torch.empty(o.shape[0] * 4, dtype=torch.float32, device="cuda")
    sc.trace_closest(rd, hd, o.shape[0], flags)
    torch.cuda.synchronize()
    h = hd.cpu().numpy().view(N.HIT_DTYPE)
    return h["prim"].copy(), h["t"].copy(), h


def core_make_rays(o, d, tmax=None):
    core = importlib.import_module("2023_render_engine_b200.core")
    return core.make_rays(o, d, tmax)


@pytest.mark.parametrize("key", ["soup1000", "soup20000", "grids"])
def test_closest_hit_matches_golden(core, gpu_ctx, key):
    g = _unpack(np.load(GOLDEN / "trace_small.npz"), key)
    sc = make_scene(core, gpu_ctx, g["v"], g["f"])
    ids, t, _ = trace_gpu(sc, g["o"], g["d"])
    assert np.array_equal(ids, g["ids"])
    hit = ids >= 0
    assert np.array_equal(t[hit], g["t"][hit])
    assert np.all(np.isinf(t[~hit]))


@pytest.mark.parametrize("nt,seed", [(2, 1), (3, 2), (4, 6), (17, 3), (513, 4), (5000, 5), (60000, 6)])
def test_closest_hit_vs_restated(core, gpu_ctx, restated, nt, seed):
    v, f = cases.soup(nt, seed, size=0.2)
    o, d = S.random_rays(20000, seed=seed + 100, lo=-1.3, hi=1.3)
    sc = make_scene(core, gpu_ctx, v, f)
    ob = restated.bvh(v, f)
    for shadow in (False, True):
        ref, tref = ob.intersect(o, d, shadow=shadow)
        ids, t, _ = trace_gpu(sc, o, d, flags=N.RT_TRACE_SHADOW if shadow else 0)
        assert np.array_equal(ids, ref)
        hit = ref >= 0
        assert np.array_equal(t[hit], tref[hit])


def test_closest_hit_edge_cases(core, gpu_ctx, restated):
    """Exact ties on shared edges/vertices, axis-aligned rays, rays starting closer to a
    surface than its error bound, transparency for shadow rays, finite tmax."""
    v, f = cases.stacked_grids()
    tr = np.zeros(f.shape[0], np.uint8)
    tr[-2:] = 1
    o, d = cases.edge_rays(9)
    sc = make_scene(core, gpu_ctx, v, f, transparent=tr)
    ob = restated.bvh(v, f, tr)
    for shadow in (False, True):
        ref, tref = ob.intersect(o, d, shadow=shadow)
        ids, t, _ = trace_gpu(sc, o, d, flags=N.RT_TRACE_SHADOW if shadow else 0)
        assert np.array_equal(ids, ref)
        assert np.array_equal(t[ref >= 0], tref[ref >= 0])
    tm = np.random.default_rng(2).uniform(0.1, 3.0, o.shape[0]).astype(np.float32)
    ref, tref = ob.intersect(o, d, tmax=tm)
    ids, t, _ = trace_gpu(sc, o, d, tmax=tm)
    assert np.array_equal(ids, ref)
    st = sc.trace_stats()
    assert st["rays"] == o.shape[0]


def test_fast_mode_agrees_on_generic_rays(core, gpu_ctx, restated):
    v, f = cases.soup(20000, 12)
    o, d = S.random_rays(50000, seed=3, lo=-1.2, hi=1.2)
    sc = make_scene(core, gpu_ctx, v, f)
    ref, _ = restated.bvh(v, f).intersect(o, d)
    ids, _, _ = trace_gpu(sc, o, d, flags=N.RT_TRACE_FAST)
    assert (ids == ref).mean() > 0.999


def test_spheres_match_reference(core, gpu_ctx):
    """Sphere::intersects arithmetic with the reference's own matrices (golden)."""
    g = np.load(GOLDEN / "spheres_cornell.npz")
    sph = [{"o2w": g[f"o2w{i}"], "w2o": g[f"w2o{i}"], "radius": float(g["radii"][i]), "glass": i == 1}
           for i in range(len(g["radii"]))]
    sc = make_scene(core, gpu_ctx, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32), spheres=sph)
    ids, t, _ = trace_gpu(sc, g["o"], g["d"])
    exp = np.where(g["ids"] >= 0, N.RT_PRIM_SHAPE | g["ids"], -1)
    assert np.array_equal(ids, exp)
    assert np.array_equal(t[ids >= 0], g["t"][g["ids"] >= 0])
    ids, t, _ = trace_gpu(sc, g["o"], g["d"], flags=N.RT_TRACE_SHADOW)
    exp = np.where(g["ids_shadow"] >= 0, N.RT_PRIM_SHAPE | g["ids_shadow"], -1)
    assert np.array_equal(ids, exp)


def test_cornell_triangles_and_spheres(core, gpu_ctx, restated):
    """Scene::intersects order: the BVH triangle first, then each shape lowers the offset."""
    g = np.load(GOLDEN / "spheres_cornell.npz")
    v, f, _, sph = cases.cornell_soup()
    spheres = [{"o2w": g[f"o2w{i}"], "w2o": g[f"w2o{i}"], "radius": float(g["radii"][i])} for i in range(2)]
    sc = make_scene(core, gpu_ctx, v, f, spheres=spheres)
    o, d = S.random_rays(20000, seed=44, lo=-0.99, hi=0.99)
    tri, ttri = restated.bvh(v, f).intersect(o, d)
    exp, texp = tri.copy(), np.where(tri >= 0, ttri, np.inf).astype(np.float32)
    for r in range(o.shape[0]):
        for i in range(2):
            hit, tt = restated.sphere_intersects(g[f"w2o{i}"], g["radii"][i], o[r], d[r], hit_offset=texp[r])
            if hit:
                exp[r], texp[r] = N.RT_PRIM_SHAPE | i, tt
    ids, t, _ = trace_gpu(sc, o, d)
    assert np.array_equal(ids, exp)
    assert np.array_equal(t[ids >= 0], texp[exp >= 0])


def test_empty_and_degenerate_inputs(core, gpu_ctx):
    import torch

    sc = make_scene(core, gpu_ctx, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32))
    o, d = S.random_rays(100, seed=1)
    ids, t, _ = trace_gpu(sc, o, d)
    assert np.all(ids == -1) and np.all(np.isinf(t))
    # zero rays
    rd = torch.empty(8, dtype=torch.float32, device="cuda")
    hd = torch.empty(4, dtype=torch.float32, device="cuda")
    sc.trace_closest(rd, hd, 0)
    # a single triangle
    v = np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0]], np.float32)
    sc1 = make_scene(core, gpu_ctx, v, np.array([[0, 1, 2]], np.uint32))
    o = np.array([[0, 0, 1], [5, 5, 1]], np.float32)
    d = np.array([[0, 0, -1], [0, 0, -1]], np.float32)
    ids, t, _ = trace_gpu(sc1, o, d)
    assert ids.tolist() == [0, -1] and t[0] == 1.0


def test_invalid_arguments_raise(core, gpu_ctx):
    sc = core.Scene(gpu_ctx)
    with pytest.raises(N.RtError):
        sc.add_mesh(np.zeros((3, 3), np.float32), np.array([[0, 1, 5]], np.uint32))
    import torch

    rd = torch.empty(8, dtype=torch.float32, device="cuda")
    hd = torch.empty(4, dtype=torch.float32, device="cuda")
    with pytest.raises(N.RtError):  # trace before commit
        sc.trace_closest(rd, hd, 1)


def test_host_buffer_entry_point(core, gpu_ctx, restated):
    v, f = cases.soup(3000, 8)
    o, d = S.random_rays(10000, seed=9, lo=-1.2, hi=1.2)
    sc = make_scene(core, gpu_ctx, v, f)
    h = sc.trace_closest_host(core_make_rays(o, d))
    ref, _ = restated.bvh(v, f).intersect(o, d)
    assert np.array_equal(h["prim"], ref)


def test_config1_full_ray_set_hash(core, gpu_ctx):
    """All 2^24 rays of the BVH-stress ray set against the reference (1.31M-triangle
    displaced icosphere in the Cornell box): the hash of every hit id and distance equals
    the hash of the reference traversal's output."""
    import torch

    info = json.loads((GOLDEN / "config1_closest_hit.json").read_text())
    sc_data = S.stress_scene()
    v, f, _ = S.flatten(sc_data)
    assert hashlib.sha256(v.tobytes()).hexdigest() == info["vertices_sha256"]
    assert hashlib.sha256(f.tobytes()).hexdigest() == info["indices_sha256"]
    o, d = S.random_rays(info["rays"], seed=info["ray_seed"])
    assert hashlib.sha256(o.tobytes()).hexdigest() == info["origins_sha256"]
    sc = make_scene(core, gpu_ctx, v, f)
    ids, t, _ = trace_gpu(sc, o, d)
    assert ids[info["sample_index"]].tolist() == info["sample_ids"]
    assert hashlib.sha256(ids.astype(np.int32).tobytes()).hexdigest() == info["ids_sha256"]
    tt = np.where(ids >= 0, t, -1.0).astype(np.float32)
    assert hashlib.sha256(tt.tobytes()).hexdigest() == info["t_sha256"]
    del torch


def test_reference_cuda_build_agrees(core, gpu_ctx):
    """The reference's own GPU traversal (its thrust path, fast-math build: the baseline in
    bench.py) returns our reference-exact ids on all but a handful of near-edge rays."""
    from oracle import bindings

    try:
        rc = bindings.RefCuda()
    except FileNotFoundError as e:
        pytest.skip(str(e))
    S_ = importlib.import_module("2023_render_engine_b200.scenes")
    v, f, _ = S_.flatten(S_.stress_scene(subdiv=5))
    o, d = S_.random_rays(1 << 18, seed=11)
    h = rc.build(v, f)
    try:
        ids, _, _ = rc.trace(h, o, d, reps=1)
    finally:
        rc.free(h)
    sc = core.Scene(gpu_ctx)
    sc.add_mesh(v, f)
    sc.commit()
    hits = sc.trace_closest_host(core.make_rays(o, d))
    assert (ids == hits["prim"]).mean() > 0.9999


def occlusion_gpu(sc, o, d, tmax, flags=0):
    """rt_trace_any (bytes) and rt_trace_any_bits for the same rays; both must agree."""
    import torch

    n = o.shape[0]
    rays = core_make_rays(o, d, tmax)
    rd = torch.from_numpy(rays.view(np.float32).reshape(-1)).cuda()
    occ = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
    bits = torch.full(((n + 31) // 32,), -1, dtype=torch.int32, device="cuda")
    sc.trace_any(rd, occ, n, flags)
    sc.trace_any_bits(rd, bits, n, flags)
    torch.cuda.synchronize()
    b = occ.cpu().numpy()
    words = bits.cpu().numpy().view(np.uint32)
    unpacked = ((words[:, None] >> np.arange(32, dtype=np.uint32)) & 1).reshape(-1).astype(np.uint8)
    assert np.array_equal(unpacked[:n], b)
    assert not unpacked[n:].any()  # bits past n are zero
    return b.astype(bool)


def distances_around(t_ref, hit, rng):
    """Light distances for the isVisible test: for rays that hit, before, exactly at, one ulp
    either side of, and beyond the reference's hit distance; for misses, anything."""
    n = t_ref.shape[0]
    pick = rng.integers(0, 6, n)
    t = np.where(hit, t_ref, 1.0).astype(np.float32)
    dist = np.select(
        [pick == 0, pick == 1, pick == 2, pick == 3, pick == 4],
        [t * np.float32(0.5), t, np.nextafter(t, np.float32(0)), np.nextafter(t, np.float32(np.inf)),
         t * np.float32(3.0)],
        rng.uniform(0.01, 5.0, n).astype(np.float32)).astype(np.float32)
    return dist


@pytest.mark.parametrize("key", ["soup1000", "soup20000", "grids"])
def test_trace_any_is_reference_isvisible(core, gpu_ctx, key):
    """rt_trace_any = Scene::isVisible's decision (Scene.cu:238-276) on the golden rays: the
    reference's closest hit along the unbounded ray, occluded when it is no farther than the
    light (visible = no hit or t > distance), with the light at, one ulp either side of, and
    away from the reference's own hit distance."""
    g = _unpack(np.load(GOLDEN / "trace_small.npz"), key)
    sc = make_scene(core, gpu_ctx, g["v"], g["f"])
    hit = g["ids"] >= 0
    dist = distances_around(g["t"], hit, np.random.default_rng(5))
    want = hit & (g["t"] <= dist)
    got = occlusion_gpu(sc, g["o"], g["d"], dist)
    assert np.array_equal(got, want)
    assert 0.2 < want.mean() < 0.8  # both answers well represented
    # any-hit mode (the renderer's shadow rays): same answer away from the boundary on generic
    # rays. On the edge rays (origins closer to the grid than its error bound) the reference's
    # offset-update quirk hides occluders behind a rejected near-zero hit (Triangle.cu:569-593):
    # there the any-hit mode may only ever report more occlusion, never less.
    fast = occlusion_gpu(sc, g["o"], g["d"], dist, N.RT_TRACE_FAST)
    away = ~hit | (np.abs(dist - g["t"]) > 1e-5 * np.maximum(g["t"], 1))
    if key == "grids":
        assert not (want & ~fast)[away].any()
    else:
        assert (fast[away] == want[away]).mean() > 0.9999


def test_trace_any_transparency_spheres_and_edges(core, gpu_ctx, restated):
    """checkShadow semantics (transparent triangles and glass spheres do not occlude), the
    analytic-shape loop of Scene::intersects and the edge rays (exact ties, axis-aligned rays,
    offsets below the error bound) with the reference's decision taken from the pinned
    restatement's closest hit."""
    g = np.load(GOLDEN / "spheres_cornell.npz")
    v, f = cases.stacked_grids()
    tr = np.zeros(f.shape[0], np.uint8)
    tr[-2:] = 1
    spheres = [{"o2w": g[f"o2w{i}"], "w2o": g[f"w2o{i}"], "radius": float(g["radii"][i]), "glass": i == 1}
               for i in range(len(g["radii"]))]
    sc = make_scene(core, gpu_ctx, v, f, transparent=tr, spheres=spheres)
    o, d = cases.edge_rays(9)
    o2, d2 = S.random_rays(20000, seed=77, lo=-1.2, hi=1.2)
    o, d = np.concatenate([o, o2]), np.concatenate([d, d2])
    rng = np.random.default_rng(8)
    ob = restated.bvh(v, f, tr)
    for shadow in (False, True):
        flags = N.RT_TRACE_SHADOW if shadow else 0
        ids, t, _ = trace_gpu(sc, o, d, flags=flags)  # closest hit, pinned to the reference elsewhere
        tri, ttri = ob.intersect(o, d, shadow=shadow)
        hit = ids >= 0
        assert np.array_equal(ids[ids < N.RT_PRIM_SHAPE], tri[ids < N.RT_PRIM_SHAPE])
        dist = distances_around(t, hit, rng)
        got = occlusion_gpu(sc, o, d, dist, flags)
        assert np.array_equal(got, hit & (t <= dist))


def test_trace_any_empty_and_invalid(core, gpu_ctx):
    import torch

    v, f = cases.soup(100, 3)
    sc = make_scene(core, gpu_ctx, v, f)
    rd = torch.zeros(8, dtype=torch.float32, device="cuda")
    occ = torch.zeros(1, dtype=torch.uint8, device="cuda")
    sc.trace_any(rd, occ, 0)
    bits = torch.zeros(2, dtype=torch.int32, device="cuda")
    with pytest.raises(N.RtError):  # a bit mask must be 4-byte aligned
        N.check(N.lib().rt_trace_any_bits(sc.handle, rd.data_ptr(), 1, bits.data_ptr() + 2, 0))


def plane_cases():
    """Planes as the reference constructs them (corner, axisX, axisY, normal): unit squares, a
    2.7 x 2.2 one (the reference truncates axis lengths to integers, Plane.cu:32-33), a tilted one
    and a glass one (transparent to shadow rays)."""
    return np.array([
        [0.5, -0.5, -0.5, 0, 1, 0, 0, 0, 1, -0.5, 0, 0],
        [-0.5, -0.5, 0.5, 1, 0, 0, 0, 1, 0, 0, 0, -0.5],
        [-1.3, -1.1, -0.9, 2.7, 0, 0, 0, 0, 2.2, 0, 1, 0],
        [-0.4, 0.3, -0.2, 0.8, 0.6, 0, -0.36, 0.48, 0.8, 0.48, -0.64, 0.6],
        [-0.5, -0.5, -0.1, 1, 0, 0, 0, 1, 0, 0, 0, 1]], np.float32)


def plane_rays(n, seed):
    """Random rays, rays aimed at the squares' interiors and edges, rays with no x component
    (the reference's offset divides by it: those never hit, Ray.cu:69-72) and grazing rays."""
    o, d = S.random_rays(n, seed=seed, lo=-1.5, hi=1.5)
    rng = np.random.default_rng(seed)
    k = n // 4
    d[:k, 0] = 0.0                                    # no x component
    d[k:2 * k, 2] = rng.uniform(-1e-6, 1e-6, k)         # grazing the z = const planes
    tgt = rng.uniform(-0.6, 0.6, (k, 3)).astype(np.float32)
    tgt[:, 2] = np.round(tgt[:, 2] * 2) / 2             # edges and corners of the unit squares
    d[2 * k:3 * k] = tgt - o[2 * k:3 * k]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return o.astype(np.float32), d.astype(np.float32)


def test_planes_match_reference(core, gpu_ctx, refo):
    """rt_scene_add_plane: closest hits of analytic planes equal the reference's own
    Plane::intersects (ids and offsets bit for bit), alone and behind a triangle mesh, in the
    order Scene::intersects tests them (Scene.cu:130-146), shadow mode included."""
    from oracle import bindings

    P = plane_cases()
    glass = np.array([0, 0, 0, 0, 1], np.uint8)
    rp = bindings.RefPlanes(refo, P, glass)
    o, d = plane_rays(40000, seed=21)
    for with_mesh in (False, True):
        sc = core.Scene(gpu_ctx)
        if with_mesh:
            v, f = cases.soup(3000, 5, size=0.15)
            sc.add_mesh(v, f)
        for j in range(len(P)):
            o2w, w2o = rp.matrices(j)
            N.check(N.lib().rt_scene_add_plane(sc.handle, o2w.ctypes.data, w2o.ctypes.data, 0, j, int(glass[j]), None))
        sc.commit()
        for shadow in (False, True):
            t0 = None
            tri = np.full(len(o), -1, np.int32)
            if with_mesh:
                rb = refo.bvh(v, f, np.zeros(f.shape[0], np.uint8))
                tri = rb.intersect(o, d, shadow=shadow)
                t0 = np.where(tri >= 0, rb.hit_t(tri, o, d), np.inf).astype(np.float32)
            pid, pt = rp.intersect(o, d, t_init=t0, shadow=shadow)
            want = np.where(pid >= 0, N.RT_PRIM_SHAPE | pid, tri)
            ids, t, h = trace_gpu(sc, o, d, flags=N.RT_TRACE_SHADOW if shadow else 0)
            assert np.array_equal(ids, want), (with_mesh, shadow, int((ids != want).sum()))
            hit = want >= 0
            assert np.array_equal(t[hit], pt[hit] if not with_mesh else np.where(pid >= 0, pt, t0)[hit])
            plane_hits = (want >= 0) & (want >= N.RT_PRIM_SHAPE)
            assert plane_hits.mean() > (0.02 if with_mesh else 0.2)
            # a plane hit reports its object-space (x, y) in the unit square
            assert np.all((h["b1"][plane_hits] >= 0) & (h["b1"][plane_hits] <= 1))
        sc.close()


def trace_counts(sc, o, d, tmax=None, flags=0):
    import torch

    rays = core_make_rays(o, d, tmax)
    rd = torch.from_numpy(rays.view(np.float32).reshape(-1)).cuda()
    cd = torch.full((2 * o.shape[0],), -1, dtype=torch.int32, device="cuda")
    sc.trace_counts(rd, cd, o.shape[0], flags)
    torch.cuda.synchronize()
    c = cd.cpu().numpy().reshape(-1, 2)
    return c[:, 0].copy(), c[:, 1].copy()


@pytest.mark.parametrize("key", ["soup1000", "soup20000", "grids"])
def test_trace_counts_invariants(core, gpu_ctx, key):
    """rt_trace_counts against what the walk must do: every ray of a non-empty scene visits the
    root and at most every node; a ray with a triangle hit tested at least one triangle; the
    any-hit walk is the closest-hit walk stopped at the first hit, so it never counts more and
    counts the same where nothing is hit; the counts are reproducible."""
    g = _unpack(np.load(GOLDEN / "trace_small.npz"), key)
    sc = make_scene(core, gpu_ctx, g["v"], g["f"])
    nnodes = sc.stats()["bvh8_nodes"]
    nodes, tris = trace_counts(sc, g["o"], g["d"])
    assert np.all(nodes >= 1) and np.all(nodes <= nnodes)
    ids, _, _ = trace_gpu(sc, g["o"], g["d"], flags=N.RT_TRACE_FAST)
    assert np.all(tris[ids >= 0] >= 1)
    an, at = trace_counts(sc, g["o"], g["d"], flags=N.RT_TRACE_COUNT_ANY)
    assert np.all(an <= nodes) and np.all(at <= tris)
    miss = ids < 0
    assert np.array_equal(an[miss], nodes[miss]) and np.array_equal(at[miss], tris[miss])
    assert np.any(an[~miss] < nodes[~miss])  # the any-hit walk does stop early
    n2, t2 = trace_counts(sc, g["o"], g["d"])
    assert np.array_equal(n2, nodes) and np.array_equal(t2, tris)


def test_trace_counts_small_and_invalid(core, gpu_ctx):
    import torch

    # one triangle: the walk is the root alone; its leaf is tested when the ray meets its box
    v = np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0]], np.float32)
    sc1 = make_scene(core, gpu_ctx, v, np.array([[0, 1, 2]], np.uint32))
    # (a ray with a zero direction component sees that axis's slab as unbounded, which keeps
    # the box test conservative: the second ray is oblique so that it misses the leaf's box)
    o = np.array([[0, 0, 1], [5, 5, 1], [0, 0, 1]], np.float32)
    d = np.array([[0, 0, -1], [0.1, 0.1, -1], [0, 0, 1]], np.float32)
    nodes, tris = trace_counts(sc1, o, d)
    assert nodes.tolist() == [1, 1, 1] and tris.tolist() == [1, 0, 0]
    # no triangles: nothing is walked
    sc0 = make_scene(core, gpu_ctx, np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32))
    nodes, tris = trace_counts(sc0, o, d)
    assert nodes.tolist() == [0, 0, 0] and tris.tolist() == [0, 0, 0]
    # zero rays is a no-op; a misaligned count buffer is refused
    rd = torch.empty(8, dtype=torch.float32, device="cuda")
    cd = torch.empty(4, dtype=torch.int32, device="cuda")
    sc1.trace_counts(rd, cd, 0)
    with pytest.raises(N.RtError):
        N.check(N.lib().rt_trace_counts(sc1.handle, rd.data_ptr(), 1, 0, cd.data_ptr() + 4))
