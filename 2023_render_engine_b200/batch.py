"""Batched multi-view rendering: autotuning and the batched-vs-individual measurement.

One rt_render_batch call renders all views of a scene in one wavefront. Two knobs are tuned:
the queue capacity (paths in flight: larger queues keep more rays per traversal launch,
smaller ones use less memory and finish the tail sooner) and the material-sort granularity
(chunk of queue slots ordered by hit material before shading: larger chunks group more lanes
by material, smaller ones keep a warp's state reads closer together). autotune times a
reduced-spp copy of the batch at each candidate and keeps the fastest.
"""
from __future__ import annotations

import time

from . import _native as N

CAPACITIES = (1 << 25, 1 << 24, 1 << 23, 1 << 22, 1 << 21)
SORT_LOG2 = (0, 8, 10, 12)


def _timed(fn, sync):
    sync()
    t0 = time.perf_counter()
    out = fn()
    sync()
    return time.perf_counter() - t0, out


def autotune_capacity(scene, views, flags, sync, candidates=CAPACITIES, probe_spp=4):
    """Fastest queue capacity for this batch, timed on a copy with spp capped at probe_spp
    (each candidate twice; the second run counts, so buffer growth is not timed).
    Returns (best capacity, [(capacity, seconds)])."""
    probe = [dict(v, spp=min(v["spp"], probe_spp)) for v in views]
    trials = []
    for cap in candidates:
        for rep in range(2):
            t, _ = _timed(lambda: scene.render_batch(probe, flags=flags, max_paths=cap), sync)
        trials.append((cap, t))
    best = min(trials, key=lambda x: x[1])[0]
    return best, trials


def autotune_sort(scene, views, flags, capacity, sync, candidates=SORT_LOG2, probe_spp=4):
    """Fastest material-sort granularity (log2 chunk, 0: off) for this batch at `capacity`,
    timed like autotune_capacity; leaves the scene set to it. Returns (best, [(log2, seconds)])."""
    probe = [dict(v, spp=min(v["spp"], probe_spp)) for v in views]
    trials = []
    for lg in candidates:
        scene.set_sort(lg)
        for rep in range(2):
            t, _ = _timed(lambda: scene.render_batch(probe, flags=flags, max_paths=capacity), sync)
        trials.append((lg, t))
    best = min(trials, key=lambda x: x[1])[0]
    scene.set_sort(best)
    return best, trials


def measure(groups, sync, autotune=True, merged=True):
    """Times every scene's views as one batch and as one rt_render call per view, and (merged)
    all views of all scenes as one batch of the merged scene.

    groups: [(name, scene, flags, views)]. Returns a dict with rays, samples and seconds of
    each way and the capacities chosen."""
    res = {"groups": [], "batched_s": 0.0, "individual_s": 0.0, "rays": 0, "samples": 0, "views": 0}
    for name, scene, flags, views in groups:
        if not views:
            continue
        cap, trials = autotune_capacity(scene, views, flags, sync) if autotune else (0, [])
        sort_log2, sort_trials = autotune_sort(scene, views, flags, cap, sync) if autotune else (10, [])
        # warm at full size: the queues grow to the batch's capacity here, not in the timed call
        scene.render_batch(views, flags=flags, max_paths=cap)
        t_b, (film, st, off) = _timed(lambda: scene.render_batch(views, flags=flags, max_paths=cap), sync)
        rays = st["extension_rays"] + st["shadow_rays"]
        del film

        def individual():
            for v in views:
                scene.render(v["camera"], spp=v["spp"], max_depth=v["max_depth"], rr_depth=v["rr_depth"],
                             seed=v["seed"], flags=flags, max_paths=cap)

        t_i, _ = _timed(individual, sync)
        samples = sum(v["camera"].width * v["camera"].height * v["spp"] for v in views)
        res["groups"].append({"scene": name, "views": len(views), "capacity": cap, "sort_log2": sort_log2,
                              "autotune": [(c, round(t, 4)) for c, t in trials],
                              "autotune_sort": [(c, round(t, 4)) for c, t in sort_trials], "batched_s": t_b,
                              "individual_s": t_i, "rays": rays, "samples": samples})
        res["batched_s"] += t_b
        res["individual_s"] += t_i
        res["rays"] += rays
        res["samples"] += samples
        res["views"] += len(views)
    res["batched_mrays_s"] = res["rays"] / res["batched_s"] / 1e6
    res["individual_mrays_s"] = res["rays"] / res["individual_s"] / 1e6
    res["batched_msamples_s"] = res["samples"] / res["batched_s"] / 1e6
    res["speedup"] = res["individual_s"] / res["batched_s"]
    if len(groups) > 1 and merged:
        res["merged"] = measure_merged(groups, sync, autotune=autotune)
        res["merged"]["speedup_vs_individual"] = res["individual_s"] / res["merged"]["seconds"]
    return res


def measure_merged(groups, sync, autotune=True):
    """All views of all groups in ONE rt_render_batch call on the merged scene (rt_scene_merge),
    its capacity and sort granularity autotuned like a group's."""
    from . import core

    scenes = [sc for _, sc, _, views in groups if views]
    flags = [fl for _, _, fl, views in groups if views]
    if any(f != flags[0] for f in flags):
        return {"unavailable": "groups render with different flags"}
    views = [dict(v, scene=k) for k, (_, _, _, vs) in enumerate([g for g in groups if g[3]]) for v in vs]
    merged = core.merge_scenes(scenes[0].ctx, scenes)
    try:
        cap, trials = autotune_capacity(merged, views, flags[0], sync) if autotune else (0, [])
        sort_log2, sort_trials = autotune_sort(merged, views, flags[0], cap, sync) if autotune else (10, [])
        merged.render_batch(views, flags=flags[0], max_paths=cap)  # warm at full size (queue growth)
        t, (film, st, _) = _timed(lambda: merged.render_batch(views, flags=flags[0], max_paths=cap), sync)
        del film
        rays = st["extension_rays"] + st["shadow_rays"]
        return {"views": len(views), "scenes": len(scenes), "capacity": cap, "sort_log2": sort_log2,
                "autotune": [(c, round(x, 4)) for c, x in trials],
                "autotune_sort": [(c, round(x, 4)) for c, x in sort_trials],
                "seconds": t, "rays": rays, "mrays_s": rays / t / 1e6, "waves": st["waves"]}
    finally:
        merged.close()


def measure_guided(scene, flags, views, guide, sync, capacity=0, train_passes=4, steps_per_pass=128,
                   batch=2 * 148 * 128):
    """The views of one scene rendered with the learned guide: `train_passes` one-spp
    recording passes over the whole batch (each followed by `steps_per_pass` training steps),
    then the batch at its own spp with the guide, against the same batch without it."""
    t0 = time.perf_counter()
    sync()
    for p in range(train_passes):
        scene.set_guide(guide, train=True)
        scene.render_batch([dict(v, spp=1, sample_offset=1000 + p) for v in views], flags=flags | N.RT_RENDER_GUIDE,
                           max_paths=capacity)
        guide.train_records(steps_per_pass, batch, seed=p)
    sync()
    t_train = time.perf_counter() - t0
    scene.set_guide(guide, train=False)
    # warm at full size: the guided queues (and the per-path mixtures) grow here, not in the timed call
    scene.render_batch(views, flags=flags | N.RT_RENDER_GUIDE, max_paths=capacity)
    t_g, (film, st, _) = _timed(lambda: scene.render_batch(views, flags=flags | N.RT_RENDER_GUIDE,
                                                           max_paths=capacity), sync)
    rays_g = st["extension_rays"] + st["shadow_rays"]
    del film
    t_p, (film, st, _) = _timed(lambda: scene.render_batch(views, flags=flags, max_paths=capacity), sync)
    rays_p = st["extension_rays"] + st["shadow_rays"]
    scene.set_guide(None)
    return {"views": len(views), "train_s": t_train, "guided_s": t_g, "plain_s": t_p,
            "guided_mrays_s": rays_g / t_g / 1e6, "plain_mrays_s": rays_p / t_p / 1e6,
            "training": {"passes": train_passes, "steps": guide.steps, "batch": batch}}
