"""Benchmark: Mrays/s of the B200 rendering core on the BVH-stress configuration.

Workload (one "step"): a full path-traced render of the BVH-stress scene (1,310,720-triangle
displaced icosphere with per-block GGX inside the Cornell box, 1,310,732 triangles) at
1920x1080, 64 samples per pixel, max depth 12, Russian roulette after depth 3, NEE on the
area light. Mrays/s = (closest-hit extension rays incl. camera rays + shadow rays) / render
time. The film (sum + count buffers) is cleared at the start of every step.

Secondary line items: closest-hit tracing of the seeded 2^24-ray BVH-stress ray set
(reference-exact ids; 512 MiB of rays, larger than the 126 MB L2), which also gives the
roofline of the dominant kernel (k_trace_closest).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun: every rank renders its own image (different seed; independent
replicas, weak scaling, no collective on the data path); the time is the max over ranks.

--impl reference times the reference renderer's own integrator (PathTracerIntegrator::render
with Scene::build and its BVH, compiled from its sources into oracle/_ref with thrust's device
system on OpenMP, so its whole render runs on this machine's host cores) on the same scene,
camera and depth; each step renders a bounded sample of the frame (a lower-resolution image of
the same view at 1 spp). Rank 0 alone runs it.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s"
WORKLOAD = ("BVH-stress render: 1920x1080, 64 spp, max depth 12, RR after depth 3, NEE on the area light; "
            "1,310,732 triangles (displaced icosphere subdiv 8, GGX F0=0.04 + Cornell box)")
TRACE_WORKLOAD = "closest hit of 2^{} seeded rays (origins uniform in [-1,1]^3, directions uniform), reference-exact ids"
NRAYS = 1 << 24
ALG_BYTES_PER_RAY = 48  # 32 B ray in + 16 B hit out (queue level)
# DRAM bytes (read + write) of one k_trace_closest launch of the 2^24-ray call: the mean of the
# four 2^24-ray launches of one ncu capture of this file's render command (1 pass, --cache-control
# none; profiles/k_trace_closest_bvh_stress.md), taken at commit 39de656 of the traversal. A
# change to traverse.cuh or trace.cu that alters k_trace_closest needs a new capture.
TRACE_TRAFFIC_BYTES_2_24 = 2_479_014_720 + 1_033_936_064


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(vals, world, device="cuda"):
    """Element-wise max of per-rank timings (every rank calls it in the same order)."""
    if world == 1:
        return [float(v) for v in vals]
    import torch

    t = torch.tensor(vals, device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t]


def rank_seed(base: int, rank: int) -> int:
    """Per-rank sample seed: every replica renders a statistically independent image."""
    return base + 97 * rank


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def build_scene(core, ctx, S):
    sc_data = S.stress_scene()
    v, f, _ = S.flatten(sc_data)
    sc = core.Scene(ctx)
    sc.add_mesh(v, f)
    sc.commit()
    return sc, v, f


def cpu_reference_rate(v, f, o, d, threads):
    """Reference traversal (oracle/_ref) over the sample; returns (Mrays/s, seconds)."""
    from oracle import bindings

    R = bindings.RefOracle()
    b = R.bvh(v, f)
    t0 = time.perf_counter()
    b.intersect(o, d, threads=threads)
    dt = time.perf_counter() - t0
    return o.shape[0] / dt / 1e6, dt


def bench_config(args):
    """The `config` both arms report: the workload this benchmark is quoted on."""
    return {"workload": WORKLOAD, "width": args.width, "height": args.height, "spp": args.spp, "max_depth": 12,
            "triangles": 1_310_732}


def reference_scene(S):
    """The BVH-stress scene in the reference harness's terms: one mesh, per-triangle materials
    (the Cornell walls, the emitter, one Trowbridge material per 64-triangle block) and the
    Cornell camera (pinhole at (0, 0, 3.5) looking down -z, 40 degree vertical field of view)."""
    from oracle import bindings

    R = bindings.RefIntegrator
    sd = S.stress_scene()
    v, f, m = S.flatten(sd)
    table = [R.entry(R.LAMBERTIAN, (0.8, 0.8, 0.8)), R.entry(R.LAMBERTIAN, (0.8, 0.1, 0.1)),
             R.entry(R.LAMBERTIAN, (0.1, 0.8, 0.1)), R.entry(R.LIGHT, (1, 1, 1), value=15.0)]
    rough = sd["roughness"]
    ggx = np.flatnonzero(m == S.MAT_GGX)
    tri_mat = m.astype(np.uint32).copy()
    for blk, r in enumerate(rough[::64][:(rough.shape[0] + 63) // 64]):
        table.append(R.entry(R.TROWBRIDGE, (1, 1, 1), (1.5, 1.5, 1.5), (0, 0, 0), (float(r), float(r))))
    tri_mat[ggx] = 4 + (np.arange(ggx.shape[0]) // 64)
    return v, f, tri_mat, table


REFERENCE_CAMERA = "camera\np 0 0 3.5\nlookat 0 0 0\nup 0 1 0\ncts 0 0 -0.8\nframeY 0.5823\n"


def reference_render_rate(host, args, S, width, height, spp, runs=1, warmup=0):
    """The reference integrator (host build, or its CUDA build) on the BVH-stress scene at
    width x height (the bench camera's view), spp, depth 12: per run (seconds in
    PathTracerIntegrator::render, rays it traced, build seconds). None if not built."""
    import tempfile

    from oracle import bindings

    try:
        R = bindings.RefIntegrator(host=host)
    except (FileNotFoundError, OSError):
        return None
    v, f, tri_mat, table = reference_scene(S)
    with tempfile.TemporaryDirectory() as td:
        cam = Path(td) / "camera.obejota"
        cam.write_text(REFERENCE_CAMERA)
        out = []
        for k in range(warmup + runs):
            _, _, _, st = R.render(cam, width, height, spp, 12, table, v, f, tri_mat)
            if k >= warmup:
                out.append(st)
    return out


def reference_config4(S, width, height, photons):
    """The reference's own integrator (host build) on the 4K photon-mapping configuration's scene:
    RENDER_MODE HYBRID with CHECK_SUBSURFACE_SCATTERING, k = 50 (MAX_NEIGHBOURS), radius 100, the
    given number of photons, at width x height (the same view), 1 spp, depth 16. Its render call
    includes its photon pass and kd-tree build (PathTracerIntegrator::render calls
    generatePhotons). None if the harness is not built."""
    import tempfile

    from oracle import bindings

    try:
        R = bindings.RefIntegrator(host=True)
    except (FileNotFoundError, OSError):
        return None
    (tv, tf), (sv, sf), spheres = S.photon_terrain(seed=11, n=1000)
    v = np.concatenate([tv, sv]).astype(np.float32)
    f = np.concatenate([tf, sf + tv.shape[0]]).astype(np.uint32)
    tri_mat = np.concatenate([np.zeros(tf.shape[0], np.uint32), np.full(sf.shape[0], 2, np.uint32)])
    tri_shape = np.concatenate([np.zeros(tf.shape[0], np.int32), np.ones(sf.shape[0], np.int32)])
    table = [R.entry(R.LAMBERTIAN, (0.6, 0.55, 0.45)), R.entry(R.DIELECTRIC, (1, 1, 1), value=1.5),
             R.subsurface_entry((0.9, 0.9, 0.9), (0.04, 0.04, 0.04), 1.3, 40.0, (1.0, 0.8, 0.6),
                                (0.01, 0.02, 0.05), 0.0)]
    sph = [(c, r, 1) for c, r in spheres]
    # the loader negates the y of every position it reads (FileImporting.cu:514-516)
    scene_file = ("camera\np 0 -2.4 5.6\nlookat 0 0.1 0\nup 0 1 0\ncts 0 0 -0.8\nframeY 0.662742\n"
                  "\nlightPoint l0\np -1.6 -2.6 1.4\nc 1 1 1\ni 50\n"
                  "\nlightPoint l1\np 1.8 -3.2 -1.2\nc 1 1 1\ni 50\n")
    R.config_photons(R.HYBRID, True, photons, 50, 100.0)
    try:
        with tempfile.TemporaryDirectory() as td:
            path = Path(td) / "config4.obejota"
            path.write_text(scene_file)
            _, _, _, st = R.render(path, width, height, 1, 16, table, v, f, tri_mat, tri_shape, spheres=sph)
    finally:
        R.config_photons(R.PATH_TRACING, False, 100000, 100, 100.0)
    rays = st["extension_rays"] + st["shadow_rays"]
    return {"workload": f"the reference's PathTracerIntegrator::render (host build) on the same scene, RENDER_MODE "
                        f"HYBRID + CHECK_SUBSURFACE_SCATTERING, {photons} photons, k = 50, {width}x{height}, 1 spp, "
                        f"depth 16; its render call includes its photon pass and kd-tree build",
            "seconds": st["render_s"], "build_s": st["build_s"], "rays": rays,
            "mrays_s": rays / st["render_s"] / 1e6, "samples_per_s": width * height / st["render_s"],
            "cores": os.cpu_count() or 1}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    S = importlib.import_module("2023_render_engine_b200.scenes")
    threads = os.cpu_count() or 1
    w, h = args.ref_width, args.ref_height
    runs = reference_render_rate(True, args, S, w, h, 1, runs=args.steps, warmup=args.warmup)
    if runs is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_integrator_host.so not built "
                                                              "(make -C oracle ref with REF_DIR set)"}))
        return
    secs = np.array([r["render_s"] for r in runs])
    rays = np.array([r["extension_rays"] + r["shadow_rays"] for r in runs], np.float64)
    ms = 1000 * float(secs.mean())
    val = float(rays.sum() / secs.sum() / 1e6)
    sample = (f"{w}x{h} image of the same view (camera, scene, depth 12), 1 spp per step; the reference's "
              f"estimator traces no shadow rays here (it has no area-light NEE)")
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": bench_config(args),
        "sample": {"rays_per_step": float(rays.mean()), "what": sample,
                   "reference_path": "PathTracerIntegrator::render + Scene::build of the reference, its BVH built "
                                     "and traversed by its own code on the host cores (thrust OpenMP system), "
                                     "shading on its 128 worker threads",
                   "build_s": float(np.mean([r["build_s"] for r in runs]))},
        "cpu_baseline": {"value": val, "unit": "Mrays/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": val, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def measure_reference_cuda(v, f, o, d, hits_d, N):
    """The reference's BVH::intersectRay on the GPU (its thrust::transform path, built with its
    own compile flags) over the same 2^24 rays: Mrays/s with the rays resident on the device,
    Mrays/s of its per-call path with host copies, and id agreement with ours."""
    try:
        from oracle import bindings

        rc = bindings.RefCuda()
    except (FileNotFoundError, OSError) as e:
        return {"unavailable": str(e)}
    t0 = time.perf_counter()
    h = rc.build(v, f)
    build_ms = (time.perf_counter() - t0) * 1e3
    try:
        ids, mk, ma = rc.trace(h, o, d, reps=3)
    finally:
        rc.free(h)
    ours = hits_d.cpu().numpy().view(N.HIT_DTYPE)["prim"]
    n = len(ids)
    return {"value": n / (mk / 1000) / 1e6, "unit": "Mrays/s", "ms_per_call": mk, "build_ms": build_ms,
            "api_value": n / (ma / 1000) / 1e6, "api_ms_per_call": ma,
            "id_agreement": float((ids == ours).mean()),
            "build": "reference BVH::intersectRay + Triangle::intersects via thrust::transform, -O3 --use_fast_math "
                     "-maxrregcount=64 (its compile.sh), sm_100a; api = its intersectRaysGpu path (rays to the "
                     "device, transform, ids back, pageable host memory)"}


def measure_scene_build(core, N, ctx, v, f, reps=3):
    """rt_scene_commit of the BVH-stress mesh: the device build (after one warm-up commit that
    loads the kernels; median of reps) and the host build (the same bytes)."""
    out = {"triangles": int(f.shape[0])}
    for name, mode, k in (("device", N.RT_BUILD_DEVICE, reps + 1), ("host", N.RT_BUILD_HOST, 1)):
        ms = []
        for _ in range(k):
            sc = core.Scene(ctx)
            sc.add_mesh(v, f)
            sc.set_build(mode)
            sc.commit()
            ms.append(sc.stats()["build_ms"])
            nodes = sc.stats()["bvh8_nodes"]
            sc.close()
        out[name + "_ms"] = float(np.median(ms[1:] if k > 1 else ms))
        out["bvh8_nodes"] = int(nodes)
    out["note"] = ("commit wall time (build + upload); both builds give the same PLOC 8-wide BVH and "
                   "reference-order tree")
    return out


def measure_guiding(args, core, N, cfgs, ctx, torch):
    """Time to RMSE <= args.guide_target on the guiding room (1280x720, max depth 16, area NEE):
    plain BSDF sampling vs the online-trained guide, against a converged FP64 render; the median
    of three runs per side."""
    GD = importlib.import_module("2023_render_engine_b200.guiding")
    sc, cam, p = cfgs.build_config2(ctx, args.guide_width, args.guide_height)
    flags = N.RT_RENDER_NEE_AREA
    t0 = time.perf_counter()
    ref = None
    per = 256
    for k in range((args.guide_ref_spp + per - 1) // per):
        ref, _ = sc.render(cam, spp=per, max_depth=p["max_depth"], rr_depth=p["rr_depth"], seed=424242, flags=flags,
                           fp64=True, film=ref, sample_offset=per * k)
    torch.cuda.synchronize()
    ref_s = time.perf_counter() - t0
    ref_mean = (ref["sum64"].view(-1, 3) / ref["count"].double().clamp_min(1).view(-1, 1))
    # warm the kernels and the guide's device buffers once (not timed), then reset the guide
    T = cfgs.GUIDE_TRAINING
    g = core.Guide(ctx, T["bbox_min"], T["bbox_max"], learning_rate=T["learning_rate"], seed=2,
                   max_depth=T["max_depth"])
    GD.render_progressive(sc, cam, g, [1, 1], max_depth=p["max_depth"], seed=7, flags=flags, train_passes=1,
                          steps_per_pass=1, batch=args.guide_batch)
    # three runs per side (fresh seeds; the guide retrained from scratch each time), the median
    # reported: one host stall inside a sub-second run would otherwise decide the comparison
    plains, guideds = [], []
    for rep in range(3):
        plains.append(GD.time_to_rmse(sc, cam, ref_mean, args.guide_target, None, pass_spp=4, max_depth=p["max_depth"],
                                      rr_depth=p["rr_depth"], seed=1 + 10 * rep, flags=flags))
        g.reset()
        guideds.append(GD.time_to_rmse(sc, cam, ref_mean, args.guide_target, g, pass_spp=4,
                                       max_depth=p["max_depth"], rr_depth=p["rr_depth"], seed=2 + 10 * rep, flags=flags,
                                       train_passes=args.guide_train_passes, steps_per_pass=args.guide_steps,
                                       batch=args.guide_batch))
    steps = g.steps
    g.close()

    def median_run(runs):
        return sorted(runs, key=lambda r: r["seconds"])[len(runs) // 2]

    plain, guided = median_run(plains), median_run(guideds)
    return {
        "metric": f"time to RMSE<={args.guide_target} vs FP64 oracle (computeRMSE), guided vs plain",
        "workload": f"guiding room {args.guide_width}x{args.guide_height}, 200k triangles, max depth 16, "
                    f"area NEE with MIS",
        "oracle": {"spp": args.guide_ref_spp, "seconds": ref_s, "estimator": "plain BSDF sampling, FP64 film"},
        "plain": {**{k: plain[k] for k in ("seconds", "spp", "rmse", "reached")},
                  "runs_seconds": [r["seconds"] for r in plains]},
        "guided": {**{k: guided[k] for k in ("seconds", "spp", "rmse", "reached")},
                   "runs_seconds": [r["seconds"] for r in guideds]},
        "speedup": (plain["seconds"] / guided["seconds"]) if guided["reached"] and plain["reached"] else None,
        "training": {"passes": args.guide_train_passes, "steps": steps, "batch": args.guide_batch,
                     "learning_rate": T["learning_rate"], "guided_depths": T["max_depth"]},
        "curves": {"plain": plain["curve"][::4], "guided": guided["curve"][::4]},
    }


def traversal_work(N, torch, sc, rays_d, n, ms=None, any_hit=False):
    """Per-ray traversal work from rt_trace_counts: BVH8 nodes visited (80 B each) and triangle
    records tested (48 B each), their bytes per ray (mean and percentiles) and, given the trace
    call's time, the rate at which the walk reads node and triangle bytes (L2 or HBM)."""
    cnt = torch.empty(2 * n, dtype=torch.int32, device="cuda")
    sc.trace_counts(rays_d, cnt, n, flags=N.RT_TRACE_COUNT_ANY if any_hit else 0)
    c = cnt.view(n, 2).to(torch.float64)
    b = 80.0 * c[:, 0] + 48.0 * c[:, 1]
    srt = torch.sort(b).values
    pick = lambda q: float(srt[min(n - 1, int(q * n))])
    out = {"rays": n, "walk": "any hit" if any_hit else "closest hit",
           "nodes_per_ray": float(c[:, 0].mean()), "triangles_per_ray": float(c[:, 1].mean()),
           "bytes_per_ray": {"mean": float(b.mean()), "p50": pick(0.5), "p90": pick(0.9), "p99": pick(0.99),
                             "max": float(srt[-1])}}
    if ms:
        out["walk_gbs"] = float(b.sum()) / (ms / 1000) / 1e9
    del cnt
    return out


def measure_traversal_work(N, torch, core, S, cfgs, ctx, sc1, rays_d, n, ms_trace):
    """bytes per ray of the walk on fixed ray sets: the 2^24-ray set of the BVH-stress scene
    (closest and any hit), and 2^20 rays with origins uniform in the bounding box of configs 0, 2
    and 4 (closest hit)."""
    res = {"config 1 (BVH stress)": traversal_work(N, torch, sc1, rays_d, n, ms=ms_trace),
           "config 1 (BVH stress), any hit": traversal_work(N, torch, sc1, rays_d, n, any_hit=True)}
    boxes = {"config 0 (Cornell box)": (cfgs.build_config0, (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)),
             "config 2 (guiding room)": (cfgs.build_config2, (-2.0, 0.0, -2.0), (2.0, 2.5, 2.0)),
             "config 4 (terrain)": (cfgs.build_config4, (-4.0, -0.4, -4.0), (4.0, 1.2, 4.0))}
    m = 1 << 20
    for name, (build, lo, hi) in boxes.items():
        sc = build(ctx)[0]
        o, d = S.random_rays(m, seed=17, lo=np.array(lo), hi=np.array(hi))
        r = torch.from_numpy(core.make_rays(o, d).view(np.float32).reshape(-1)).cuda()
        res[name] = traversal_work(N, torch, sc, r, m)
        sc.close()
        del r
    return res


def measure_guide_inference(core, cfgs, ctx, torch, stream, rows):
    """rt_guide_eval on `rows` seeded queries (positions in the guiding room's box, unit normals
    and directions): the network forward on the tensor cores (tcgen05), encoding and output
    stores included. Inputs (36 B/row) and outputs (192 B/row) exceed L2 at 2^21 rows."""
    T = cfgs.GUIDE_TRAINING
    g = core.Guide(ctx, T["bbox_min"], T["bbox_max"], learning_rate=T["learning_rate"], seed=3)
    rng = np.random.default_rng(11)
    lo, hi = np.asarray(T["bbox_min"], np.float64), np.asarray(T["bbox_max"], np.float64)
    n = rng.normal(size=(rows, 3))
    w = rng.normal(size=(rows, 3))
    q = np.concatenate([rng.uniform(lo, hi, size=(rows, 3)), n / np.linalg.norm(n, axis=1, keepdims=True),
                        w / np.linalg.norm(w, axis=1, keepdims=True)], 1).astype(np.float32)
    qd = torch.from_numpy(q.reshape(-1)).cuda()
    for _ in range(3):
        g.eval(qd)
    ms = []
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.eval(qd)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    g.close()
    t = float(np.mean(ms))
    flops = 49_776.0 * rows  # 2 x (144*64 + 3*64*64 + 64*48) multiply-adds per row
    tf = flops / (t * 1e-3) / 1e12
    pf = ROOT / "MEASURED_PEAKS.json"
    peak = float(json.loads(pf.read_text())["bf16_tflops"]) if pf.exists() else 1590.0
    return {"workload": f"rt_guide_eval of {rows} rows (144 -> 64 x4 -> 48, FP16 operands, FP32 accumulation)",
            "ms": t, "rows_per_s": rows / (t * 1e-3), "network_tflops": tf,
            "tensor_frac": tf / peak, "tensor_peak": peak,
            "tensor_peak_kind": "measured bf16 burst" if pf.exists() else "fallback",
            "bytes_per_row": 36 + 192, "gbs": rows * 228 / (t * 1e-3) / 1e9}


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    core = importlib.import_module("2023_render_engine_b200.core")
    S = importlib.import_module("2023_render_engine_b200.scenes")
    N = importlib.import_module("2023_render_engine_b200._native")
    cfgs = importlib.import_module("2023_render_engine_b200.configs")
    dev = torch.cuda.current_device()
    ctx = core.Context(dev)
    stream = torch.cuda.Stream()  # a stream of its own: the default stream cannot be captured
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    sc, cam, p = cfgs.build_config1(ctx, args.width, args.height)
    v, f, _ = S.flatten(S.stress_scene())
    W, H = cam.width, cam.height
    film = {"sum": torch.zeros(H * W * 3, dtype=torch.float32, device="cuda"),
            "count": torch.zeros(H * W, dtype=torch.int32, device="cuda")}
    host_sum = torch.empty(H * W * 3, dtype=torch.float32).pin_memory()
    host_cnt = torch.empty(H * W, dtype=torch.int32).pin_memory()
    # --host-wave-loop: the host checks the queues after every 4-wave group (a profiling aid: ncu
    # does not see kernels inside the device loop's conditional graph); the same kernels and rays
    rflags = N.RT_RENDER_NEE_AREA | (N.RT_RENDER_HOST_LOOP if args.host_wave_loop else 0)

    def render_step(seed):
        film["sum"].zero_()
        film["count"].zero_()
        _, st = sc.render(cam, spp=args.spp, max_depth=p["max_depth"], rr_depth=p["rr_depth"], seed=seed,
                          flags=rflags, film=film)
        return st

    # ---- render, film resident on the device
    for w in range(args.warmup):
        render_step(rank_seed(1000 + w, rank))
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    rays = []
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        for k in range(args.steps):
            st = render_step(rank_seed(k, rank))
            rays.append(st["extension_rays"] + st["shadow_rays"])
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    rays_step = float(np.mean(rays))
    st_last = st

    # ---- end to end: the render call + the film read back into pinned host memory
    torch.cuda.synchronize()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        render_step(rank_seed(500 + k, rank))
        host_sum.copy_(film["sum"], non_blocking=True)
        host_cnt.copy_(film["count"], non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = e0.elapsed_time(e1) / args.steps

    # ---- one more frame (untimed) with its stages timed by CUDA events: where the frame goes
    film["sum"].zero_()
    film["count"].zero_()
    _, st_stages = sc.render(cam, spp=args.spp, max_depth=p["max_depth"], rr_depth=p["rr_depth"],
                             seed=rank_seed(900, rank), flags=rflags | N.RT_RENDER_STAGE_TIMES, film=film)
    stage_ms = {k: round(v, 3) for k, v in sc.stage_times().items()}
    stage_ms["frame"] = round(st_stages["ms"], 3)

    # ---- closest-hit trace of the 2^24-ray set (dominant kernel, roofline)
    o, d = S.random_rays(NRAYS, seed=7 + rank)
    rays_np = core.make_rays(o, d)
    rays_d = torch.from_numpy(rays_np.view(np.float32).reshape(-1)).cuda()
    hits_d = torch.empty(NRAYS * 4, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        sc.trace_closest(rays_d, hits_d, NRAYS)
    torch.cuda.synchronize()
    barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        sc.trace_closest(rays_d, hits_d, NRAYS)
    t1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_trace = t0.elapsed_time(t1) / args.steps
    fallback = sc.trace_stats()["exact_fallback_rays"]
    # the same rays in RT_TRACE_FAST mode (the renderer's extension rays: no reference-order checks)
    for _ in range(2):
        sc.trace_closest(rays_d, hits_d, NRAYS, N.RT_TRACE_FAST)
    torch.cuda.synchronize()
    t0.record(stream)
    for _ in range(args.steps):
        sc.trace_closest(rays_d, hits_d, NRAYS, N.RT_TRACE_FAST)
    t1.record(stream)
    torch.cuda.synchronize()
    ms_trace_fast = t0.elapsed_time(t1) / args.steps
    sc.trace_closest(rays_d, hits_d, NRAYS)  # the reference-exact hits again (compared further down)
    trav_work = None
    if world == 1 and not args.no_traversal_work:
        trav_work = measure_traversal_work(N, torch, core, S, cfgs, ctx, sc, rays_d, NRAYS, ms_trace)

    # ---- learned guiding: time to RMSE <= target against the FP64 converged render, guided vs
    # plain, on the guiding room (one process only: it is a sequence of dependent passes)
    guiding = None
    if world == 1 and args.guide_ref_spp > 0:
        guiding = measure_guiding(args, core, N, cfgs, ctx, torch)
    guide_inference = None
    if world == 1 and args.guide_eval_rows > 0:
        guide_inference = measure_guide_inference(core, cfgs, ctx, torch, stream, args.guide_eval_rows)

    # ---- batched multi-view rendering (64 views of configs 0-2, one wavefront per scene)
    batched = None
    if world == 1 and not args.no_batch:
        B = importlib.import_module("2023_render_engine_b200.batch")
        groups = cfgs.build_config3(ctx, n_views=64, seed=5)
        batched = B.measure(groups, torch.cuda.synchronize)
        T = cfgs.GUIDE_TRAINING
        name, sc2, fl2, views2 = groups[2]
        g = core.Guide(ctx, T["bbox_min"], T["bbox_max"], learning_rate=T["learning_rate"], seed=2,
                       max_depth=T["max_depth"])
        batched["guided"] = B.measure_guided(sc2, fl2, views2, g, torch.cuda.synchronize,
                                             capacity=batched["groups"][2]["capacity"])
        batched["guided"]["scene"] = name
        g.close()
        batched["workload"] = ("64 views drawn from configs 0-2 (seeded poses; resolution log-uniform 128^2-1024^2, "
                               "aspect 0.5-2; spp in {4..64}; depth 8-16), area NEE; one rt_render_batch per "
                               "scene vs one rt_render per view")
        del groups

    # ---- photon mapping + subsurface scattering + guiding at 4K (config 4)
    photon_sss = None
    if world == 1 and args.c4_spp > 0:
        PR = importlib.import_module("2023_render_engine_b200.photon_render")
        photon_sss = PR.measure(ctx, torch, stream, width=args.c4_width, height=args.c4_height, spp=args.c4_spp)
        photon_sss["metric"] = ("Mrays/s, samples/s and photon-map gathers/s of hybrid + subsurface rendering; "
                                "guided vs plain time to equal noise")
        if not args.no_cpu_baseline:
            photon_sss["reference"] = reference_config4(S, args.c4_ref_width, args.c4_ref_height, args.c4_ref_photons)

    # ---- the reference's own CUDA traversal on the same rays (baseline, not a target)
    ref_cuda = None
    if world == 1 and not args.no_ref_cuda:
        ref_cuda = measure_reference_cuda(v, f, o, d, hits_d, N)
        runs = reference_render_rate(False, args, S, args.ref_width, args.ref_height, 1, runs=2, warmup=1)
        if runs:
            secs = sum(r["render_s"] for r in runs)
            rays_ref = sum(r["extension_rays"] + r["shadow_rays"] for r in runs)
            ref_cuda["render"] = {
                "value": rays_ref / secs / 1e6, "unit": "Mrays/s",
                "workload": f"the reference's PathTracerIntegrator::render, its stock CUDA build (compile.sh flags: "
                            f"BVH built and traversed on this GPU by thrust, shading on its host threads), on the "
                            f"same scene and view at {args.ref_width}x{args.ref_height}, 1 spp, depth 12",
                "rays_per_run": rays_ref / len(runs), "seconds_per_run": secs / len(runs)}

    # ---- scene commit: device vs host build of the same structures
    scene_build = measure_scene_build(core, N, ctx, v, f) if world == 1 else None
    if scene_build is not None and ref_cuda is not None:
        scene_build["reference_ms"] = ref_cuda["build_ms"]

    ms, ms_e2e, ms_trace = max_over_ranks([ms, ms_e2e, ms_trace], world)
    if rank == 0:
        peak, peak_kind = measured_peaks()
        rate = rays_step * world / (ms / 1000) / 1e6
        rate_e2e = rays_step * world / (ms_e2e / 1000) / 1e6
        trace_rate = NRAYS * world / (ms_trace / 1000) / 1e6
        achieved = NRAYS * ALG_BYTES_PER_RAY / (ms_trace / 1000) / 1e9
        samples = W * H * args.spp
        line = {
            "metric": METRIC, "value": rate, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene, camera and sample streams)",
            "config": bench_config(args),
            "details": {"rays_per_step_per_gpu": rays_step,
                        "extension_rays": int(st_last["extension_rays"]), "shadow_rays": int(st_last["shadow_rays"]),
                        "camera_rays": int(st_last["camera_rays"]), "waves": int(st_last["waves"]),
                        "samples_per_s": samples * world / (ms / 1000),
                        "l2": "scene ~140 MB and path queues ~1 GB per step exceed the 126 MB L2",
                        "parallelism": f"replicas x{world}",
                        "stage_ms": stage_ms},
            "e2e": {"value": rate_e2e, "unit": "Mrays/s", "h2d_bytes_per_step": 144 + 32,
                    "d2h_bytes_per_step": W * H * 16,
                    "note": "render call through the C ABI + film read back to pinned host memory; the inputs "
                            "of a step are the camera and options structs"},
            "trace": {"workload": TRACE_WORKLOAD.format(NRAYS.bit_length() - 1), "value": trace_rate, "unit": "Mrays/s", "ms_per_step": ms_trace,
                      "exact_fallback_rays": int(fallback),
                      "fast_value": NRAYS * world / (ms_trace_fast / 1000) / 1e6, "fast_ms_per_step": ms_trace_fast},
            # per frame: 6 kernels a wave (closest hit, its replay, material sort, shade, shadow,
            # retire), the wave check of each 4-wave group and the first camera rays
            "gpu_launches": args.steps * (int(st_last["waves"]) * 6 + (int(st_last["waves"]) + 3) // 4 + 1),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": (TRACE_TRAFFIC_BYTES_2_24 / (ms_trace / 1000) / 1e9) if NRAYS == 1 << 24 else None,
                         "traffic_bytes_per_launch": TRACE_TRAFFIC_BYTES_2_24 if NRAYS == 1 << 24 else None,
                         "kernel": "k_trace_closest (2^24-ray closest-hit call, 48 B/ray queue-level bytes)",
                         # what the walk itself reads (nodes x 80 B + triangle records x 48 B per ray, counted
                         # by rt_trace_counts), over the same launch time: mostly L1 and L2 hits
                         "walk": ({"bytes_per_ray": trav_work["config 1 (BVH stress)"]["bytes_per_ray"]["mean"],
                                   "gbs": trav_work["config 1 (BVH stress)"]["walk_gbs"],
                                   "frac_of_hbm_peak": trav_work["config 1 (BVH stress)"]["walk_gbs"] / peak}
                                  if trav_work else None),
                         "note": f"peak {peak_kind}; traffic (GB/s over the same launch time) from the ncu capture "
                                 "of the full launch: 4.4x the algorithmic bytes, the scene re-read past L2 and the "
                                 "traversal stacks in local memory; see profiles/"},
            "clocks": clk.summary(),
            "traversal_work": trav_work,
            "guiding": guiding,
            "guide_inference": guide_inference,
            "reference_cuda": ref_cuda,
            "batched": batched,
            "photon_sss": photon_sss,
            "scene_build": scene_build,
        }
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            w, h = args.ref_width, args.ref_height
            runs = reference_render_rate(True, args, S, w, h, 1, runs=1)
            if runs:
                r = runs[0]
                rays_ref = r["extension_rays"] + r["shadow_rays"]
                line["cpu_baseline"] = {
                    "value": rays_ref / r["render_s"] / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "reference",
                    "sample": f"the reference's PathTracerIntegrator::render on the same scene and view at {w}x{h}, "
                              f"1 spp, depth 12 ({rays_ref} rays in {r['render_s']:.1f} s; BVH built and traversed "
                              f"by its own code on the host cores)"}
            ns = args.cpu_sample
            val, dt = cpu_reference_rate(v, f, o[:ns], d[:ns], threads)
            line["cpu_baseline_traversal"] = {
                "value": val, "unit": "Mrays/s", "cores": threads, "kind": "reference",
                "sample": f"first {ns} rays of the BVH-stress ray set through the reference's BVH::intersectRay "
                          f"({dt:.1f} s); traversal only", "ours": trace_rate}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=1 << 20)
    ap.add_argument("--ref-width", type=int, default=960, help="reference integrator sample image width")
    ap.add_argument("--ref-height", type=int, default=540)
    ap.add_argument("--rays-log2", type=int, default=24, help="smaller ray sets for profiler captures")
    ap.add_argument("--host-wave-loop", action="store_true",
                    help="render with the host-side wave loop (profiler captures of the render kernels)")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--guide-ref-spp", type=int, default=4096, help="0 skips the guiding measurement")
    ap.add_argument("--no-ref-cuda", action="store_true", help="skip the reference CUDA traversal baseline")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched multi-view measurement")
    ap.add_argument("--no-traversal-work", action="store_true", help="skip the per-ray traversal work counts")
    ap.add_argument("--c4-spp", type=int, default=256, help="config-4 spp per mode (0 skips config 4)")
    ap.add_argument("--c4-width", type=int, default=3840)
    ap.add_argument("--c4-height", type=int, default=2160)
    ap.add_argument("--c4-ref-width", type=int, default=384, help="reference config-4 sample image width")
    ap.add_argument("--c4-ref-height", type=int, default=216)
    ap.add_argument("--c4-ref-photons", type=int, default=1_000_000, help="photons of the reference config-4 sample")
    ap.add_argument("--guide-target", type=float, default=0.01)
    ap.add_argument("--guide-width", type=int, default=1280)
    ap.add_argument("--guide-height", type=int, default=720)
    ap.add_argument("--guide-train-passes", type=int, default=4)
    ap.add_argument("--guide-steps", type=int, default=128, help="Adam steps per recording pass "
                    "(configs.GUIDE_TRAINING)")
    ap.add_argument("--guide-batch", type=int, default=2 * 148 * 128, help="samples per Adam step "
                    "(configs.GUIDE_TRAINING: one round of the training kernel's tiles on 148 SMs)")
    ap.add_argument("--guide-eval-rows", type=int, default=1 << 21, help="guide inference rows (0 skips)")
    args = ap.parse_args()
    global NRAYS
    NRAYS = 1 << args.rays_log2
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
