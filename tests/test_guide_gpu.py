"""Path guide on the GPU against its CPU oracle (oracle/guide_oracle.py): network outputs,
mixture density, sampling, the training gradient and the Adam step; then the guide inside the
path tracer: training-record bookkeeping, unbiasedness of the one-sample MIS estimator and the
gain of the trained guide over BSDF sampling."""
import importlib

import numpy as np
import pytest

from oracle import guide_oracle as G

pytestmark = pytest.mark.gpu

N = importlib.import_module("2023_render_engine_b200._native")
S = importlib.import_module("2023_render_engine_b200.scenes")
C = importlib.import_module("2023_render_engine_b200.configs")
GD = importlib.import_module("2023_render_engine_b200.guiding")

BMIN, BMAX = np.array([-2.0, 0.0, -2.0], np.float32), np.array([2.0, 2.5, 2.0], np.float32)


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def batch(rng, B):
    p = rng.uniform(BMIN, BMAX, size=(B, 3))
    q = np.concatenate([p, unit(rng.normal(size=(B, 3))), unit(rng.normal(size=(B, 3)))], 1).astype(np.float32)
    wi = unit(rng.normal(size=(B, 3))).astype(np.float32)
    pdfb = rng.uniform(0.05, 1.0, size=B).astype(np.float32)
    w = rng.lognormal(0.0, 1.0, size=B).astype(np.float32)
    return q, wi, pdfb, w


def cuda(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32).reshape(-1)).cuda()


@pytest.fixture()
def guide(core, gpu_ctx):
    g = core.Guide(gpu_ctx, BMIN, BMAX, learning_rate=1e-2, seed=7)
    yield g
    g.close()


@pytest.mark.parametrize("B", [1, 3000, 100003])
def test_eval_matches_oracle(guide, B):
    """Row counts that are not a multiple of the 128-row tile; 100003 rows give every
    persistent CTA several tiles (the completion barrier's phase alternates across them)."""
    rng = np.random.default_rng(B)
    q, _, _, _ = batch(rng, B)
    out = guide.eval(cuda(q)).cpu().numpy()
    _, ref = G.forward(guide.params(), G.encode(q, BMIN, BMAX))
    assert np.all(np.isfinite(out))
    err = np.abs(out - ref)
    assert err.mean() < 2e-3 * np.abs(ref).mean() + 1e-4
    assert np.allclose(out, ref, atol=3e-2, rtol=3e-2)


def test_pdf_matches_oracle(guide):
    rng = np.random.default_rng(1)
    q, wi, pdfb, _ = batch(rng, 4096)
    pdf = guide.pdf(cuda(q), cuda(wi), cuda(pdfb)).cpu().numpy()
    _, out = G.forward(guide.params(), G.encode(q, BMIN, BMAX))
    ref = G.mixture_pdf(out, wi, pdfb)
    assert np.allclose(pdf, ref, rtol=2e-2, atol=1e-4)


def fib_sphere(m):
    i = np.arange(m) + 0.5
    z = 1 - 2 * i / m
    r = np.sqrt(1 - z * z)
    ph = np.pi * (1 + 5 ** 0.5) * i
    return np.stack([r * np.cos(ph), r * np.sin(ph), z], 1)


def cube_face(d):
    a = np.argmax(np.abs(d), 1)
    return a * 2 + (d[np.arange(len(d)), a] > 0)


def test_sample_matches_oracle_and_density(guide):
    rng = np.random.default_rng(2)
    nq, reps = 6, 1 << 15
    q, _, _, _ = batch(rng, nq)
    qq = np.repeat(q, reps, axis=0)
    u = rng.uniform(size=(qq.shape[0], 3)).astype(np.float32)
    dirs, pdf = guide.sample(cuda(qq), cuda(u))
    dirs, pdf = dirs.cpu().numpy().astype(np.float64), pdf.cpu().numpy()
    assert np.allclose(np.linalg.norm(dirs, axis=1), 1, atol=1e-4)
    out = guide.eval(cuda(q)).cpu().numpy()
    # the same uniforms through the oracle give the same directions (a lobe pick may differ
    # where u0 falls on a lobe boundary)
    ref = G.sample(np.repeat(out, reps, axis=0), u)
    assert (np.linalg.norm(dirs - ref, axis=1) < 2e-2).mean() > 0.99
    # the returned density is the mixture's at the sample
    dec = G.decode(np.repeat(out, reps, axis=0))
    assert np.allclose(pdf, G.guide_pdf(dec, dirs), rtol=2e-3, atol=1e-6)
    # and the samples follow it: per cube face, sample frequency vs quadrature of the density
    fib = fib_sphere(1 << 21)
    ff = cube_face(fib)
    for b in range(nq):
        hist = np.bincount(cube_face(dirs[b * reps:(b + 1) * reps]), minlength=6) / reps
        d1 = {k: v[b:b + 1].repeat(len(fib), 0) for k, v in G.decode(out).items()}
        p = G.guide_pdf(d1, fib)
        expect = np.array([(p * (ff == k)).mean() * 4 * np.pi for k in range(6)])
        assert np.allclose(hist, expect, atol=0.015), (b, hist, expect)


def test_gradient_matches_oracle(guide):
    rng = np.random.default_rng(3)
    q, wi, pdfb, w = batch(rng, 5000)
    loss, grad = guide.train_step(cuda(q), cuda(wi), cuda(pdfb), cuda(w), apply=False, want_grad=True)
    ref_loss, ref = G.loss_and_grad(guide.params(), q, wi, pdfb, w, BMIN, BMAX, fp16=True)
    assert guide.steps == 0
    assert abs(loss - ref_loss) <= 1e-3 * abs(ref_loss)
    assert np.linalg.norm(grad - ref) / np.linalg.norm(ref) < 1e-2
    for l, (wo, bo) in enumerate(G.OFFSETS):  # every layer's weights and biases
        e = bo + G.layer_out(l)
        assert np.linalg.norm(grad[wo:e] - ref[wo:e]) / np.linalg.norm(ref[wo:e]) < 3e-2, l
    # deterministic: the same batch gives the same bits
    _, grad2 = guide.train_step(cuda(q), cuda(wi), cuda(pdfb), cuda(w), apply=False, want_grad=True)
    assert np.array_equal(grad, grad2)


def test_adam_step_matches_oracle(guide):
    rng = np.random.default_rng(4)
    q, wi, pdfb, w = batch(rng, 2048)
    p0 = guide.params()
    _, grad = guide.train_step(cuda(q), cuda(wi), cuda(pdfb), cuda(w), apply=True, want_grad=True)
    p1 = guide.params()
    ref, _, _ = G.adam(p0, np.zeros_like(p0), np.zeros_like(p0), grad, 1, 1e-2)
    assert guide.steps == 1
    assert np.allclose(p1, ref, rtol=1e-5, atol=1e-7)
    # the FP16 image follows the master weights: outputs match the oracle on the new weights
    out = guide.eval(cuda(q[:512])).cpu().numpy()
    _, r = G.forward(p1, G.encode(q[:512], BMIN, BMAX))
    _, r0 = G.forward(p0, G.encode(q[:512], BMIN, BMAX))
    assert np.allclose(out, r, atol=3e-2, rtol=3e-2)
    assert np.abs(out - r).mean() < 0.2 * np.abs(out - r0).mean()


def test_set_params_roundtrip_resets_adam(guide):
    rng = np.random.default_rng(5)
    p = (guide.params() * 0.5).astype(np.float32)
    guide.set_params(p)
    assert np.array_equal(guide.params(), p)
    assert guide.steps == 0
    with pytest.raises(Exception):
        guide.set_params(p[:-1])


def test_training_fits_a_direction_field(core, gpu_ctx):
    """Online-learning check: incident light from a position-dependent direction (towards a
    point source) — the trained mixture concentrates there."""
    import torch

    g = core.Guide(gpu_ctx, BMIN, BMAX, learning_rate=1e-2, seed=1)
    rng = np.random.default_rng(6)
    src = np.array([0.5, 2.2, 1.5])
    B = 1 << 14
    loss0 = None
    for it in range(300):
        q, _, _, _ = batch(rng, B)
        d = unit(src - q[:, :3])
        # samples of the integrand: around d with a few degrees of spread, weight 1; BSDF pdf uniform
        wi = unit(d + 0.05 * rng.normal(size=d.shape)).astype(np.float32)
        loss, _ = g.train_step(cuda(q), cuda(wi), cuda(np.full(B, 1 / (4 * np.pi))), cuda(np.ones(B)))
        if loss0 is None:
            loss0 = loss
    qt, _, _, _ = batch(rng, 4096)
    dt = unit(src - qt[:, :3]).astype(np.float32)
    p_at = g.pdf(cuda(qt), cuda(dt), cuda(np.full(4096, 1 / (4 * np.pi)))).cpu().numpy()
    p_away = g.pdf(cuda(qt), cuda(-dt), cuda(np.full(4096, 1 / (4 * np.pi)))).cpu().numpy()
    assert loss < loss0 - 2.0
    assert np.median(p_at) > 20.0 / (4 * np.pi)
    assert np.median(p_at / p_away) > 100
    g.close()
    del torch


def walls_scene(core, ctx):
    """Cornell walls and ceiling light only: every scattering vertex is Lambertian."""
    d = S.cornell_box()
    sc = core.Scene(ctx)
    sc.set_materials(C.cornell_materials())
    for v, f, m in d["meshes"]:
        sc.add_mesh(v, f, material=m)
    sc.commit()
    return sc


def test_record_bookkeeping(core, gpu_ctx):
    """Without NEE every contribution after a path's first guided vertex lands in that vertex's
    record, so the sum of first-record suffix radiance equals the film total minus the emission
    seen directly by the camera (same seed, depth-1 render)."""
    sc = walls_scene(core, gpu_ctx)
    cam = C.cornell_camera(64, 64)
    g = core.Guide(gpu_ctx, [-1.01] * 3, [1.01] * 3, seed=3)
    sc.set_guide(g, train=True)
    film, _ = sc.render(cam, spp=4, max_depth=8, seed=11, flags=N.RT_RENDER_GUIDE, fp64=True)
    direct, _ = sc.render(cam, spp=4, max_depth=1, seed=11, fp64=True)
    rec = g.records()
    n, nnz = g.record_count()
    assert n > 64 * 64 * 4 and 0 < nnz <= n
    prev = rec[:, 19].view(np.uint32)
    first = prev == 0x3FFFFF
    assert np.all((prev < np.arange(n)) | first)
    total = film["sum64"].double().sum().item() - direct["sum64"].double().sum().item()
    got = rec[first, 16:19].astype(np.float64).sum()
    assert abs(got - total) <= 1e-4 * abs(total)
    # the training weight of a record is S / beta; nonzero exactly where S > 0
    w = (rec[:, 16:19] / np.maximum(rec[:, 13:16], 1e-30)).mean(1)
    assert (w > 0).sum() == nnz
    g.close()


def tile_means(film, core, W, H, t):
    img = core.film_mean(film).reshape(H, W, 3)
    return img.reshape(H // t, t, W // t, t, 3).mean(axis=(1, 3))


@pytest.mark.parametrize("nee", [False, True])
def test_guided_estimator_unbiased(core, gpu_ctx, nee):
    """Cornell box (with the glass sphere): the guided image equals the BSDF-sampled image in
    expectation, per 4x4 tile (z-test over independent repeats)."""
    sc, cam, _ = C.build_config0(gpu_ctx, 32, 32)
    g = core.Guide(gpu_ctx, [-1.01] * 3, [1.01] * 3, seed=5)
    flags = N.RT_RENDER_NEE_AREA if nee else 0
    GD.render_progressive(sc, cam, g, [4, 4, 4, 4], max_depth=8, seed=100, flags=flags, train_passes=4,
                          steps_per_pass=8, batch=1 << 14)
    assert g.steps == 32
    K = 8
    guided, plain = [], []
    for k in range(K):
        sc.set_guide(g, train=False)
        f, _ = sc.render(cam, spp=64, max_depth=8, seed=1000 + k, flags=flags | N.RT_RENDER_GUIDE)
        guided.append(tile_means(f, core, 32, 32, 4))
        f, _ = sc.render(cam, spp=64, max_depth=8, seed=2000 + k, flags=flags)
        plain.append(tile_means(f, core, 32, 32, 4))
    guided, plain = np.array(guided), np.array(plain)
    diff = guided.mean(0) - plain.mean(0)
    se = np.sqrt(guided.var(0, ddof=1) / K + plain.var(0, ddof=1) / K) + 1e-9
    z = np.abs(diff / se)
    assert np.mean(z > 3.5) < 0.01, (z.max(), np.mean(z > 3.5))
    assert abs(guided.mean() / plain.mean() - 1) < 0.01
    g.close()


def test_trained_guide_lowers_error(core, gpu_ctx):
    """Light through a gap in a wall (mostly indirect): after online training, the guided
    estimator's error against a converged render is lower than BSDF sampling's at equal spp."""
    sc, cam, cfg = C.build_config2(gpu_ctx, 512, 288)
    flags = N.RT_RENDER_NEE_AREA
    ref = None
    for k in range(8):
        ref, _ = sc.render(cam, spp=256, max_depth=16, seed=9, flags=flags, fp64=True, film=ref, sample_offset=256 * k)
    T = C.GUIDE_TRAINING
    g = core.Guide(gpu_ctx, T["bbox_min"], T["bbox_max"], learning_rate=T["learning_rate"], seed=2)
    try:
        GD.render_progressive(sc, cam, g, [1] * 8, max_depth=16, seed=300, flags=flags, train_passes=8,
                              steps_per_pass=32, batch=1 << 16)
        errs_g, errs_p = [], []
        for k in range(6):
            sc.set_guide(g, train=False)
            fg, _ = sc.render(cam, spp=64, max_depth=16, seed=500 + k, flags=flags | N.RT_RENDER_GUIDE)
            fp, _ = sc.render(cam, spp=64, max_depth=16, seed=600 + k, flags=flags)
            errs_g.append(core.rmse(fg, ref))
            errs_p.append(core.rmse(fp, ref))
        # measured ratio at this size: 0.90-0.97 across runs (the training batches come from
        # records appended in arrival order, so runs differ); the six-seed means scatter by ~1%
        assert np.mean(errs_g) < 0.98 * np.mean(errs_p), (errs_g, errs_p)
        assert max(errs_g) < min(errs_p) * 1.02, (errs_g, errs_p)
    finally:
        sc.set_guide(None)
        g.close()
