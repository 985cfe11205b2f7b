"""Progressive guided rendering: online training of the path guide on the tracer's own samples.

Each pass renders `spp` samples per pixel into the same film (distinct sample indices, so the
passes are independent); during the first `train_passes` passes the tracer records every guided
vertex and the guide takes Adam steps on those records after the pass. Sampling uses the guide
from the first pass after its first step (before that the guided vertices sample the BSDF).
"""
from __future__ import annotations

import time

from . import _native as N


def pass_schedule(total_spp: int, first: int = 1, growth: float = 2.0, cap: int = 64):
    """Pass sizes: first, first*growth, ... capped at `cap`, summing to total_spp."""
    out, done, s = [], 0, first
    while done < total_spp:
        k = min(int(s), cap, total_spp - done)
        out.append(k)
        done += k
        s = s * growth
    return out


def render_progressive(scene, camera, guide, passes, max_depth: int, rr_depth: int = 3, seed: int = 0,
                       flags: int = 0, train_passes: int = 0, steps_per_pass: int = 4, batch: int = 1 << 18,
                       film=None, fp64: bool = False, on_pass=None, sync=None):
    """Renders len(passes) passes (passes[i] spp each); guided when `guide` is not None.

    on_pass(i, spp_done, film, seconds) is called after each pass (its own time is not
    counted); `sync` is a callable that waits for the device (torch.cuda.synchronize).
    Returns (film, seconds spent rendering and training)."""
    total_s = 0.0
    done = 0
    for i, spp in enumerate(passes):
        if sync:
            sync()
        t0 = time.perf_counter()
        f = flags
        if guide is not None:
            train = i < train_passes
            scene.set_guide(guide, train=train)
            f |= N.RT_RENDER_GUIDE
        film, _ = scene.render(camera, spp=spp, max_depth=max_depth, rr_depth=rr_depth, seed=seed, flags=f,
                               sample_offset=done, film=film, fp64=fp64)
        if guide is not None and i < train_passes:
            _, nnz = guide.record_count()
            if nnz:
                guide.train_records(steps_per_pass, batch, seed=seed * 7919 + i)
        if sync:
            sync()
        total_s += time.perf_counter() - t0
        done += spp
        if on_pass is not None:
            on_pass(i, done, film, total_s)
    if guide is not None:
        scene.set_guide(guide, train=False)
    return film, total_s


def film_rmse(film, ref_mean) -> float:
    """computeRMSE (camera/Film.cu:611-632) of a device film against a device (H*W, 3) float64
    mean image: sqrt(sum over pixels of the squared RGB difference / pixels)."""
    s = (film["sum64"] if "sum64" in film else film["sum"]).double().view(-1, 3)
    c = film["count"].double().clamp_min(1).view(-1, 1)
    d = s / c - ref_mean
    return float((d * d).sum().sqrt().item() / (ref_mean.shape[0] ** 0.5))


def time_to_rmse(scene, camera, ref_mean, target: float, guide=None, pass_spp: int = 4, max_spp: int = 4096,
                 max_depth: int = 16, rr_depth: int = 3, seed: int = 0, flags: int = 0, train_passes: int = 0,
                 steps_per_pass: int = 32, batch: int = 1 << 16):
    """Renders progressively until the RMSE against `ref_mean` reaches `target`.

    Plain (guide None): passes of `pass_spp`. Guided: first `train_passes` passes of 1 spp, each
    followed by `steps_per_pass` training steps on its records, then passes of `pass_spp` with
    the trained guide. The clock (device-synchronised) covers rendering and training, not the
    RMSE checks. Returns dict(seconds, spp, rmse, reached, curve)."""
    import torch

    passes = [1] * train_passes if guide is not None else []
    while sum(passes) < max_spp:
        passes.append(pass_spp)
    curve = []
    state = {"done": False}

    class _Stop(Exception):
        pass

    def on_pass(i, spp, film, seconds):
        e = film_rmse(film, ref_mean)
        curve.append((spp, seconds, e))
        if e <= target:
            raise _Stop()

    try:
        render_progressive(scene, camera, guide, passes, max_depth=max_depth, rr_depth=rr_depth, seed=seed,
                           flags=flags, train_passes=train_passes, steps_per_pass=steps_per_pass, batch=batch,
                           on_pass=on_pass, sync=torch.cuda.synchronize)
    except _Stop:
        state["done"] = True
        if guide is not None:
            scene.set_guide(guide, train=False)
    spp, seconds, e = curve[-1]
    return {"seconds": seconds, "spp": spp, "rmse": e, "reached": state["done"], "curve": curve}


def profile_passes(width: int = 1280, height: int = 720, guided_passes: int = 2, pass_spp: int = 4):
    """The guiding room's schedule with the host-side wave loop, for profiler launch lists (ncu
    does not list the kernels inside the device loop's conditional graph): the training passes
    (one spp, then the configured Adam steps), then `guided_passes` pairs of a guided and a plain
    pass of `pass_spp`. Every render call starts with one k_start launch."""
    import torch

    from . import configs, core

    torch.cuda.set_device(0)
    ctx = core.Context(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    sc, cam, _ = configs.build_config2(ctx, width, height)
    flags = N.RT_RENDER_NEE_AREA | N.RT_RENDER_HOST_LOOP
    T = configs.GUIDE_TRAINING
    g = core.Guide(ctx, T["bbox_min"], T["bbox_max"], learning_rate=T["learning_rate"], seed=2,
                   max_depth=T["max_depth"])
    sc.set_guide(g, train=True)
    for i in range(T["train_passes"]):
        sc.render(cam, spp=1, max_depth=16, rr_depth=3, seed=7 + i, flags=flags | N.RT_RENDER_GUIDE)
        g.train_records(T["steps_per_pass"], T["batch"], seed=i)
    sc.set_guide(g, train=False)
    for k in range(guided_passes):
        sc.render(cam, spp=pass_spp, max_depth=16, rr_depth=3, seed=100 + k, flags=flags | N.RT_RENDER_GUIDE)
        sc.render(cam, spp=pass_spp, max_depth=16, rr_depth=3, seed=200 + k, flags=flags)
    torch.cuda.synchronize()


if __name__ == "__main__":
    profile_passes()
