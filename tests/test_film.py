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


@pytest.mark.parametrize("w,h", [(1, 1), (5, 3), (6, 2), (7, 9), (48, 48)])
def test_bmp_and_ppm_writers_match_reference_layout(core, refr, tmp_path, w, h):
    """rt_image_write_bmp against the reference's BitmapImage::write_image on the same pixels
    (odd widths exercise the row padding and the quirky image-size field); the PPM header."""
    rng = np.random.default_rng(w * 31 + h)
    rgb = rng.integers(0, 256, size=(h * w, 3), dtype=np.uint8)
    core.image_write(tmp_path / "ours.bmp", rgb, w, h, "bmp")
    bgr_rows = rgb.reshape(h, w, 3)[::-1, :, ::-1]  # file row i = film row h - 1 - i, BGR
    refr.bmp_write(tmp_path / "ref.bmp", bgr_rows, w, h)
    assert (tmp_path / "ours.bmp").read_bytes() == (tmp_path / "ref.bmp").read_bytes()
    core.image_write(tmp_path / "ours.ppm", rgb, w, h, "ppm")
    assert (tmp_path / "ours.ppm").read_bytes() == f"P6\n{w} {h}\n255\n".encode() + rgb.tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", range(6))
@pytest.mark.parametrize("fmt", ["bmp", "ppm"])
def test_tonemap_files_match_reference(core, refr, tmp_path, mode, fmt):
    """rt_film_tonemap + the writers against Film::writeToBMP / writeToPPM on the same sums
    (FP64 film): identical files, except that gammaClamp's pow may round a value that lands
    within an ulp of a byte boundary the other way."""
    import torch

    rng = np.random.default_rng(100 + mode)
    npix = refr.width * refr.height
    s = random_sums(rng, npix)
    s[:40] *= 1e4  # values above the white point: uncharted2 goes past 1 (not clamped)
    samples = 16
    film = {"sum64": torch.from_numpy(s.reshape(-1)).cuda(),
            "count": torch.full((npix,), samples, dtype=torch.int32, device="cuda"),
            "sum": torch.zeros(npix * 3, dtype=torch.float32, device="cuda")}
    rgb = core.film_tonemap(film, samples, mode).cpu().numpy()
    ours = tmp_path / f"ours.{fmt}"
    core.image_write(ours, rgb, refr.width, refr.height, fmt)
    refr.film_write(tmp_path / "ref", s, samples, mode, bmp=(fmt == "bmp"))
    a = np.frombuffer(ours.read_bytes(), np.uint8)
    b = np.frombuffer((tmp_path / f"ref.{fmt}").read_bytes(), np.uint8)
    assert a.shape == b.shape
    diff = np.nonzero(a != b)[0]
    if mode == N.RT_TONEMAP_GAMMA_CLAMP:
        assert diff.size <= 3 and np.all(np.abs(a[diff].astype(int) - b[diff].astype(int)) == 1), diff
    else:
        assert diff.size == 0, (diff[:10], a[diff[:10]], b[diff[:10]])
