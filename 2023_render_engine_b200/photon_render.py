"""Photon mapping + subsurface scattering + guiding at 4K (config 4), measured end to end.

The steps are the reference's photon pipeline (Scene::generatePhotons + computePhotons, the
kd-tree build, then PathTracerIntegrator::render with the photon estimates,
integration/Scene.cu:989-1026, 607-722, 914-969) on the GPU:

1. trace the photons from the two point lights (rt_photons_trace);
2. build the kd-tree over them (rt_photon_map_build);
3. render in hybrid + subsurface mode with k-nearest-photon density gathers at every
   scattering vertex and dipole gathers at camera hits on the slab — plain BSDF sampling, and
   with a guide trained online on the same scene first.

Each render is timed with CUDA events on the context's stream; Mrays/s counts extension and
shadow rays, and the gather rate counts photon-map estimates. A render is two halves with
disjoint sample indices in two films, so that their difference measures the image noise of
each mode without a converged reference at 4K.
"""
from __future__ import annotations

import importlib
import time

from . import _native as N
from . import configs, core

GD = importlib.import_module(__package__ + ".guiding")


def _event_ms(torch, stream, fn):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


def measure(ctx, torch, stream, width=3840, height=2160, spp=None, photons=None, k=None, seed=11,
            guided=True, train_passes=4, train_steps=128, train_batch=2 * 148 * 128, terrain_n=1000):
    """Runs config 4 once and returns a dict of its timings and rates."""
    spp = spp or 256
    photons = photons or configs.CONFIG4_PHOTONS
    k = k or configs.CONFIG4_K
    t0 = time.perf_counter()
    sc, cam, p = configs.build_config4(ctx, width, height, seed=seed, n=terrain_n)
    build_s = time.perf_counter() - t0
    stats = sc.stats()
    fl = configs.CONFIG4_FLAGS
    out = {"workload": f"config 4: {stats['triangles']} triangles (displaced terrain) + 16 glass spheres + "
                       f"subsurface slab, 2 point lights; {photons} photons, k={k}; {width}x{height}, {spp} spp, "
                       f"max depth {p['max_depth']}, hybrid + subsurface",
           "scene_build_s": build_s}

    # warm the photon and render kernels on a small case (not timed)
    pm_w, _ = sc.trace_photons(100_000, max_depth=16, seed=seed + 100)
    pm_w.build()
    sc.set_photon_map(pm_w, k, 100.0)
    small = core.look_at_camera((0.0, 2.4, 5.6), (0.0, -0.1, 0.0), (0, 1, 0), 45.0, 64, 36)
    sc.render(small, spp=1, max_depth=p["max_depth"], seed=1, flags=fl)
    torch.cuda.synchronize()

    # 1. photon trace. The call allocates the new map's buffers before its kernels run; its own
    # event-timed figure (pst["ms"]) covers the kernels, the outer one the allocations too, which
    # vary with how much device memory the process already holds
    ms_call, (pm, pst) = _event_ms(torch, stream, lambda: sc.trace_photons(photons, max_depth=16, seed=seed + 1))
    ms_trace = pst["ms"]
    out["photon_trace"] = {"ms": ms_trace, "ms_with_allocation": ms_call, "emitted": int(pst["emitted"]),
                           "stored": len(pm), "rays": int(pst["rays"]),
                           "emitted_per_s": pst["emitted"] / (ms_trace / 1000),
                           "Mrays_per_s": pst["rays"] / (ms_trace / 1000) / 1e6}
    # 2. kd-tree (host build over the device photons, then upload)
    t0 = time.perf_counter()
    pm.build()
    out["kd_build_s"] = time.perf_counter() - t0
    sc.set_photon_map(pm, k, 100.0)
    pm_w.close()

    W, H = cam.width, cam.height
    half = max(spp // 2, 1)
    films = [{"sum": torch.zeros(H * W * 3, dtype=torch.float32, device="cuda"),
              "count": torch.zeros(H * W, dtype=torch.int32, device="cuda")} for _ in range(2)]

    def render_halves(flags, rseed):
        """spp samples per pixel as two halves with disjoint sample indices, into two films;
        returns the device time of both, their stats summed, and the noise estimate of the
        full-spp image: RMSE(half a, half b) / 2 (each half has sqrt(2) times the noise of the
        whole, and their difference sqrt(2) times that again)."""
        for f in films:
            f["sum"].zero_()
            f["count"].zero_()
        total = {}
        ms = 0.0
        for h, f in enumerate(films):
            t, (_, st) = _event_ms(torch, stream, lambda: sc.render(
                cam, spp=half, max_depth=p["max_depth"], rr_depth=p["rr_depth"], seed=rseed, flags=flags,
                sample_offset=h * half, film=f))
            ms += t
            for key, v in st.items():
                total[key] = total.get(key, 0) + v
        return ms, total, core.film_rmse_gpu(films[0], films[1]) / 2.0

    def line(ms, st, noise):
        rays = st["extension_rays"] + st["shadow_rays"]
        return {"ms": ms, "Mrays_per_s": rays / (ms / 1000) / 1e6, "samples_per_s": W * H * 2 * half / (ms / 1000),
                "gathers_per_s": st["gathers"] / (ms / 1000), "extension_rays": int(st["extension_rays"]),
                "shadow_rays": int(st["shadow_rays"]), "gathers": int(st["gathers"]), "waves": int(st["waves"]),
                "noise_rmse": noise}

    # 3a. plain
    out["plain"] = line(*render_halves(fl, 5))
    if guided:
        T = configs.CONFIG4_GUIDE
        g = core.Guide(ctx, T["bbox_min"], T["bbox_max"], learning_rate=T["learning_rate"], seed=2,
                       max_depth=T["max_depth"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        GD.render_progressive(sc, cam, g, [1] * train_passes, max_depth=p["max_depth"], rr_depth=p["rr_depth"],
                              seed=77, flags=fl, train_passes=train_passes, steps_per_pass=train_steps,
                              batch=train_batch, sync=torch.cuda.synchronize)
        out["guide_training_s"] = time.perf_counter() - t0
        out["guide_training"] = {"passes": train_passes, "steps": g.steps, "batch": train_batch,
                                 "learning_rate": T["learning_rate"], "guided_depths": T["max_depth"]}
        sc.set_guide(g, train=False)
        # 3b. guided
        out["guided"] = line(*render_halves(fl | N.RT_RENDER_GUIDE, 6))
        sc.set_guide(None)
        g.close()
        pl, gd = out["plain"], out["guided"]
        if gd["noise_rmse"] > 0 and gd["ms"] > 0:
            # time to equal error, plain over guided (error^2 falls as 1/time), training included
            out["guided_efficiency"] = (pl["noise_rmse"] ** 2 * pl["ms"]) / (
                gd["noise_rmse"] ** 2 * (gd["ms"] + 1000 * out["guide_training_s"]))
    sc.set_photon_map(None)
    pm.close()
    sc.close()
    return out


def main(argv=None):
    """Command line: one config-4 measurement on cuda:0, printed as JSON."""
    import argparse
    import json

    import torch

    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--width", type=int, default=3840)
    ap.add_argument("--height", type=int, default=2160)
    ap.add_argument("--spp", type=int, default=256)
    ap.add_argument("--photons", type=int, default=configs.CONFIG4_PHOTONS)
    ap.add_argument("--plain", action="store_true", help="skip the guided render")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    ctx = core.Context(0)
    stream = torch.cuda.Stream()  # a stream of its own: the default stream cannot be captured
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    r = measure(ctx, torch, stream, width=a.width, height=a.height, spp=a.spp, photons=a.photons,
                guided=not a.plain)
    print(json.dumps(r, indent=1), flush=True)


if __name__ == "__main__":
    main()
