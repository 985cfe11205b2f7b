"""rt_trace_closest_noalloc: the closest-hit trace for callers that cannot allocate device
memory while tracing (a render thread on a frame budget, or a host whose own allocator owns
all device memory). Its scratch is a fixed array inside the library, shared by all calls.

This file is collected last so that a run stopping at the first failure has already run
every other test; it also passes on its own in a fresh process."""
import ctypes
import importlib

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu

N = importlib.import_module("2023_render_engine_b200._native")
S = importlib.import_module("2023_render_engine_b200.scenes")


def _trace(fn, sc, rays_d, hits_d, n, flags=0):
    import torch

    hits_d.fill_(-7.0)  # stale values must not leak into the result
    N.check(fn(sc.handle, rays_d.data_ptr(), n, hits_d.data_ptr(), flags))
    torch.cuda.synchronize()
    return hits_d.cpu().numpy().view(N.HIT_DTYPE).copy()


def test_noalloc_matches_allocating_entry_point(core, gpu_ctx):
    import torch

    lib = N.lib()
    v, f = cases.stacked_grids()
    v2, f2 = cases.soup(20000, 12)
    sc = core.Scene(gpu_ctx)
    sc.add_mesh(v, f)
    sc.add_mesh(v2, f2)
    sc.commit()
    for call, (n, seed) in enumerate([(50000, 31), (1 << 20, 32)]):  # two calls in a row, the second at the limit
        o, d = S.random_rays(n, seed=seed, lo=-1.3, hi=1.3)
        if call == 0:  # exact ties, zero direction components, near-zero offsets
            eo, ed = cases.edge_rays(4)
            o[: len(eo)], d[: len(ed)] = eo, ed
        rays_d = torch.from_numpy(core.make_rays(o, d).view(np.float32).reshape(-1)).cuda()
        hits_d = torch.empty(n * 4, dtype=torch.float32, device="cuda")
        for flags in (0, N.RT_TRACE_SHADOW):
            ref = _trace(lib.rt_trace_closest, sc, rays_d, hits_d, n, flags)
            ref_stats = sc.trace_stats()
            got = _trace(lib.rt_trace_closest_noalloc, sc, rays_d, hits_d, n, flags)
            got_stats = sc.trace_stats()
            assert np.array_equal(got["prim"], ref["prim"])
            hit = ref["prim"] >= 0
            assert np.array_equal(got["t"][hit], ref["t"][hit])
            assert np.array_equal(got["b1"][hit], ref["b1"][hit])
            assert np.array_equal(got["b2"][hit], ref["b2"][hit])
            # the replay queue half of the shared array carried the same rays
            assert got_stats == ref_stats
            if call == 0:
                assert got_stats["exact_fallback_rays"] > 0
    # an empty call after calls that left counters behind reports nothing of theirs
    N.check(lib.rt_trace_closest_noalloc(sc.handle, rays_d.data_ptr(), 0, hits_d.data_ptr(), 0))
    assert sc.trace_stats() == {"rays": 0, "exact_fallback_rays": 0}


def test_noalloc_rejects_batches_above_the_limit(core, gpu_ctx):
    import torch

    sc = core.Scene(gpu_ctx)
    v, f = cases.soup(100, 1)
    sc.add_mesh(v, f)
    sc.commit()
    n = (1 << 20) + 1
    rays_d = torch.zeros(n * 8, dtype=torch.float32, device="cuda")
    hits_d = torch.zeros(n * 4, dtype=torch.float32, device="cuda")
    st = N.lib().rt_trace_closest_noalloc(sc.handle, rays_d.data_ptr(), n, hits_d.data_ptr(), 0)
    assert st == 7  # RT_ERR_CAPACITY
    assert "1048576" in N.last_error()
