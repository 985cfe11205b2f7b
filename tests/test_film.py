"""Film accumulation files (.hdrbmp) and computeRMSE against the reference's own Film
(camera/Film.cu:366-449, 611-632, compiled into oracle/_ref/libref_render.so). CPU: the
loader and the RMSE formula; GPU: the writer and the GPU RMSE on rendered films."""
import importlib

import numpy as np
import pytest

N = importlib.import_module("2023_render_engine_b200._native")


@pytest.fixture(scope="module")
def refr():
    from oracle import bindings

    try:
        return bindings.RefRender()
    except FileNotFoundError as e:
        pytest.skip(str(e))


def random_sums(rng, npix):
    mag = 10.0 ** rng.uniform(-6, 3, size=(npix, 1))
    s = rng.uniform(0, 1, size=(npix, 3)) * mag
    s[rng.uniform(size=npix) < 0.05] = 0.0
    return s


def test_loader_reads_reference_files(core, refr, tmp_path):
    rng = np.random.default_rng(0)
    s = random_sums(rng, refr.width * refr.height)
    path = tmp_path / "ref"
    refr.film_store(path, s, 37)
    ref_sums, ref_n = refr.film_load(path)
    ours, n = core.film_load_hdrbmp(path, refr.width, refr.height)
    assert n == ref_n == 37
    assert np.array_equal(ours, ref_sums)
    assert np.allclose(ours, s, rtol=1e-5, atol=0)  # six significant digits in the file
    with pytest.raises(Exception):
        core.film_load_hdrbmp(path, refr.width + 1, refr.height)


def test_rmse_formula_matches_compute_rmse(core, refr):
    rng = np.random.default_rng(1)
    a, b = random_sums(rng, refr.width * refr.height), random_sums(rng, refr.width * refr.height)
    got = core.rmse(a / 16, b / 64)
    assert abs(got - refr.film_rmse(a, 16, b, 64)) <= 1e-6 * got  # computeRMSE returns a float


@pytest.mark.gpu
def test_writer_and_gpu_rmse_match_reference(core, gpu_ctx, refr, tmp_path):
    cfg = importlib.import_module("2023_render_engine_b200.configs")
    sc, cam, p = cfg.build_config0(gpu_ctx, refr.width, refr.height)
    fa, _ = sc.render(cam, spp=8, max_depth=8, seed=1, flags=N.RT_RENDER_NEE_AREA, fp64=True)
    fb, _ = sc.render(cam, spp=8, max_depth=8, seed=2, flags=N.RT_RENDER_NEE_AREA)
    path = tmp_path / "ours"
    core.film_store_hdrbmp(path, fa, refr.width, refr.height, 8)
    ref_sums, n = refr.film_load(path)
    want = core.film_mean(fa) * 8
    assert n == 8
    assert np.allclose(ref_sums, want, rtol=1e-5, atol=1e-300)
    # the same sums written by the reference give the same bytes
    refr.film_store(tmp_path / "theirs", want, 8)
    assert (tmp_path / "ours.hdrbmp").read_bytes() == (tmp_path / "theirs.hdrbmp").read_bytes()
    # GPU computeRMSE against the reference's on the same films
    got = core.film_rmse_gpu(fa, fb)
    ref = refr.film_rmse(core.film_mean(fa) * 8, 8, core.film_mean(fb) * 8, 8)
    assert abs(got - ref) <= 1e-6 * ref  # computeRMSE returns a float
