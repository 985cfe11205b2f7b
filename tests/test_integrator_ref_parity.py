"""Parity with the reference's OWN integrator and materials on scenes with triangle meshes,
spheres, glass and area emitters (oracle/ref_integrator_harness.cu: PathTracerIntegrator::render
with Scene::build and its BVH, compiled from its sources with thrust's device system on OpenMP,
so the reference renders triangle scenes on the host cores).

* Dielectric (glass) and mirror sampling against DielectricMaterial / MirrorMaterial
  (DielectricMaterial.cu:59-77: refraction with probability 0.7 else reflection, no division by
  the lobe probability; fresnelDielectric, geometricMath.cu:203-239, with its quirks).
* Images at equal samples per pixel, per 4x4-pixel tile, with a z-test whose variance comes from
  independent runs of each side (the reference seeds its sampler from std::random_device):
  the Cornell box of the Cornell configuration (10 triangles of Lambertian walls, a 2-triangle
  area emitter hit by paths, a Lambertian sphere and a glass sphere), and a variant with a
  Trowbridge floor, a Trowbridge sphere and a point light (next-event estimation with the
  reference's delta-light MIS weight, shadow rays through glass)."""
import importlib
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = importlib.import_module("2023_render_engine_b200._native")
S = importlib.import_module("2023_render_engine_b200.scenes")
cfgs = importlib.import_module("2023_render_engine_b200.configs")

CAMERA = textwrap.dedent("""\
    camera
    p 0 0 3.5
    lookat 0 0 0
    up 0 1 0
    cts 0 0 -0.8
    frameY 0.5823
    """)


@pytest.fixture(scope="module")
def refi():
    from oracle import bindings

    try:
        return bindings.RefIntegrator(host=True)
    except FileNotFoundError as e:
        pytest.skip(str(e))


def unit(a):
    return (a / np.linalg.norm(a, axis=-1, keepdims=True)).astype(np.float32)


def ref_entry(R, m):
    """The harness's table entry for one of our rt_material values."""
    c = tuple(m.color)
    if m.type == N.RT_MAT_LAMBERTIAN:
        return R.entry(R.LAMBERTIAN, c)
    if m.type == N.RT_MAT_TROWBRIDGE:
        return R.entry(R.TROWBRIDGE, c, tuple(m.eta), tuple(m.k), tuple(m.roughness))
    if m.type == N.RT_MAT_LIGHT:
        return R.entry(R.LIGHT, c, value=m.intensity)
    if m.type == N.RT_MAT_DIELECTRIC:
        return R.entry(R.DIELECTRIC, c, value=m.ior)
    if m.type == N.RT_MAT_MIRROR:
        return R.entry(R.MIRROR, c)
    raise ValueError(m.type)


@pytest.mark.parametrize("kind", ["dielectric", "mirror"])
def test_specular_sampling_matches_reference_classes(core, refi, kind):
    """For each outgoing direction the reference's two glass lobes are deterministic: both
    sides must give the same directions and values (refraction 1 - F, reflection F with the
    reference's Fresnel; 0 under total internal reflection), and pick refraction with
    probability 0.7."""
    if kind == "dielectric":
        mat = core.material(N.RT_MAT_DIELECTRIC, color=(0.9, 0.8, 0.7), ior=1.5, transparent=True)
    else:
        mat = core.material(N.RT_MAT_MIRROR, color=(0.9, 0.8, 0.7))
    entry = ref_entry(refi, mat)
    rng = np.random.default_rng(4)
    ncase, reps = 300, 64
    wo = unit(rng.normal(size=(ncase, 3)))
    wo[:20, 2] = rng.uniform(-0.02, 0.02, 20)  # grazing, both sides
    wo[20:40] = unit(np.column_stack([rng.normal(size=(20, 2)), -rng.uniform(0.01, 0.3, 20)]))  # inside, near TIR
    wo = unit(wo)
    # reference: every case under `reps` seeds -> its refraction and reflection results
    rw, rv, ru = refi.material_sample(entry, np.repeat(wo, reps, 0), np.arange(ncase * reps))
    rw, rv, ru = rw.reshape(ncase, reps, 3), rv.reshape(ncase, reps, 3), ru.reshape(ncase, reps)
    gw, gv, _, gdelta = core.material_sample(mat, np.repeat(wo, reps, 0), seed=9, flags=N.RT_RENDER_COMPAT)
    gw, gv = gw.reshape(ncase, reps, 3), gv.reshape(ncase, reps, 3)
    assert gdelta.all()
    refr_ref = refr_ours = total = 0
    for i in range(ncase):
        lobes = {}
        for j in range(reps):
            lobe = "t" if (kind == "dielectric" and ru[i, j] < 0.7) else "r"
            lobes.setdefault(lobe, (rw[i, j], rv[i, j]))
        for j in range(reps):
            v = gv[i, j]
            matched = None
            for lobe, (w_ref, v_ref) in lobes.items():
                same_value = np.allclose(v, v_ref, rtol=1e-5, atol=1e-6)
                if np.all(v_ref == 0):  # total internal reflection: the reference leaves wi unset
                    if same_value:
                        matched = lobe
                elif same_value and np.allclose(gw[i, j], w_ref, atol=2e-6):
                    matched = lobe
            assert matched is not None, (i, wo[i], gw[i, j], v, lobes)
            refr_ours += matched == "t"
        refr_ref += int((ru[i] < 0.7).sum()) if kind == "dielectric" else 0
        total += reps
    if kind == "dielectric":
        p_ref, p_ours = refr_ref / total, refr_ours / total
        sigma = np.sqrt(0.7 * 0.3 / total)
        assert abs(p_ref - 0.7) < 5 * sigma and abs(p_ours - 0.7) < 5 * sigma


def tiles(img, w, h, t=4):
    return img.reshape(h // t, t, w // t, t, 3).mean(axis=(1, 3)).reshape(-1, 3)


def z_stats(ref_imgs, my_imgs, w, h):
    R = np.stack([tiles(i, w, h) for i in ref_imgs])
    M = np.stack([tiles(i, w, h) for i in my_imgs])
    runs_r, runs_m = R.shape[0], M.shape[0]
    se = np.sqrt(R.var(axis=0, ddof=1) / runs_r + M.var(axis=0, ddof=1) / runs_m)
    z = (M.mean(0) - R.mean(0)) / np.maximum(se, 1e-12)
    zs = z[se > 0]
    return zs, abs(M.mean() - R.mean()) / R.mean()


def cornell_scene(core, trowbridge_variant):
    """(our material table, meshes, spheres, point lights) of the Cornell box or its variant."""
    mats = cfgs.cornell_materials()
    walls = S.cornell_walls()
    meshes = [(v, f, m) for (v, f), m in walls.values()]
    spheres = [(s["center"], s["radius"], s["material"]) for s in S.cornell_box()["spheres"]]
    lights = []
    if trowbridge_variant:
        # a Trowbridge floor (roughness 0.25), a smoother Trowbridge sphere, a point light
        mats.append(core.material(N.RT_MAT_TROWBRIDGE, color=(0.9, 0.9, 0.9), eta=(1.5, 1.5, 1.5), k=(0, 0, 0),
                                  roughness=(0.1, 0.1)))
        names = list(walls.keys())
        meshes = [(v, f, S.MAT_GGX if names[k] == "floor" else m) for k, (v, f, m) in enumerate(meshes)]
        spheres = [(spheres[0][0], spheres[0][1], len(mats) - 1), spheres[1]]
        lights = [((0.0, 0.3, 0.2), (1.0, 0.9, 0.8), 1.5)]
    return mats, meshes, spheres, lights


def render_both(core, gpu_ctx, refi, tmp_path, trowbridge_variant, w=64, h=64, spp=16, depth=8, runs=8):
    mats, meshes, spheres, lights = cornell_scene(core, trowbridge_variant)
    # the loader negates the y of every position it reads (FileImporting.cu:514-516)
    obj = CAMERA + "".join(f"\nlightPoint l{i}\np {p[0]} {-p[1]} {p[2]}\nc {c[0]} {c[1]} {c[2]}\ni {s}\n"
                           for i, (p, c, s) in enumerate(lights))
    path = tmp_path / "scene.obejota"
    path.write_text(obj)
    # one vertex array for the reference's single mesh, per-triangle materials and shape ids
    vs, fs, ms, ss = [], [], [], []
    base = 0
    for k, (v, f, m) in enumerate(meshes):
        vs.append(v)
        fs.append(f + base)
        ms.append(np.full(f.shape[0], m, np.uint32))
        ss.append(np.full(f.shape[0], k, np.int32))
        base += v.shape[0]
    V, F, M, SH = np.concatenate(vs), np.concatenate(fs), np.concatenate(ms), np.concatenate(ss)
    table = [ref_entry(refi, m) for m in mats]
    ref_imgs, c2w, r2c = [], None, None
    for _ in range(runs):
        img, c2w, r2c, st = refi.render(path, w, h, spp, depth, table, V, F, M, SH, spheres=spheres)
        ref_imgs.append(img)
        assert st["extension_rays"] > w * h * spp
    sc = core.Scene(gpu_ctx)
    sc.set_materials(mats)
    for k, (v, f, m) in enumerate(meshes):
        sc.add_mesh(v, f, material=m, shape_id=k)
    for j, (c, r, m) in enumerate(spheres):
        o2w, w2o = S.sphere_matrices(c, r)
        sc.add_sphere(o2w, w2o, r, material=m, shape_id=100 + j, transparent=mats[m].type == N.RT_MAT_DIELECTRIC)
    for p, c, s in lights:
        sc.add_point_light(p, c, s)
    sc.commit()
    cam = N.Camera()
    cam.camera_to_world[:] = [float(x) for x in c2w.reshape(-1)]
    cam.raster_to_camera[:] = [float(x) for x in r2c.reshape(-1)]
    cam.lens_radius, cam.focal_distance, cam.width, cam.height = 0.0, 0.0, w, h
    my_imgs = []
    for r in range(runs):
        film, _ = sc.render(cam, spp=spp, max_depth=depth, rr_depth=3, seed=300 + r, flags=N.RT_RENDER_COMPAT,
                            fp64=True)
        my_imgs.append(core.film_mean(film))
    return ref_imgs, my_imgs, w, h


@pytest.mark.parametrize("variant", ["cornell", "trowbridge_point_light"])
def test_image_parity_with_reference_integrator(core, gpu_ctx, refi, tmp_path, variant):
    ref_imgs, my_imgs, w, h = render_both(core, gpu_ctx, refi, tmp_path, variant != "cornell")
    zs, rel = z_stats(ref_imgs, my_imgs, w, h)
    assert np.abs(zs).mean() < 1.2, np.abs(zs).mean()     # ~0.8 expected under equal means
    assert (np.abs(zs) > 4).mean() < 0.01
    assert abs(zs.mean()) < 0.25, zs.mean()
    assert rel < 0.02, rel


def test_photon_pass_matches_reference_generate_photons(core, gpu_ctx, refi, tmp_path):
    """rt_photons_trace against the reference's own photon pass (generatePhotons,
    photonDispersion.cu:175-192, Scene::generatePhotons, Scene.cu:989-1018) on the Cornell box
    (Lambertian walls and sphere, a glass sphere photons pass through) lit by a point light:
    the number of stored photons per emitted photon, their total power and the power and count
    landing on each shape agree within the run-to-run spread (independent runs of each side,
    z within 4)."""
    mats, meshes, spheres, _ = cornell_scene(core, False)
    light = ((0.0, 0.5, -0.1), (1.0, 0.9, 0.8), 2.0)
    path = tmp_path / "photons.obejota"
    p, c, i = light
    path.write_text(CAMERA + f"\nlightPoint l0\np {p[0]} {-p[1]} {p[2]}\nc {c[0]} {c[1]} {c[2]}\ni {i}\n")
    vs, fs, ms, ss = [], [], [], []
    base = 0
    for k, (v, f, m) in enumerate(meshes):
        vs.append(v)
        fs.append(f + base)
        ms.append(np.full(f.shape[0], m, np.uint32))
        ss.append(np.full(f.shape[0], 10 + k, np.int32))  # spheres are shapes 0 and 1 in the reference
        base += v.shape[0]
    V, F, M, SH = np.concatenate(vs), np.concatenate(fs), np.concatenate(ms), np.concatenate(ss)
    table = [ref_entry(refi, m) for m in mats]
    n, runs = 100_000, 6
    shapes = [0, 1] + [10 + k for k in range(len(meshes))]

    def summary(power, shape):
        row = [len(shape) / n, *(power.sum(0) / n)]
        for s in shapes:
            sel = shape == s
            row += [sel.sum() / n, power[sel].sum() / n]
        return np.array(row)

    ref_rows = []
    for _ in range(runs):
        _, pw, sh = refi.photons(path, n, table, V, F, M, SH, spheres=spheres)
        ref_rows.append(summary(pw.astype(np.float64), sh))
    sc = core.Scene(gpu_ctx)
    sc.set_materials(mats)
    for k, (v, f, m) in enumerate(meshes):
        sc.add_mesh(v, f, material=m, shape_id=10 + k)
    for j, (cc, r, m) in enumerate(spheres):
        o2w, w2o = S.sphere_matrices(cc, r)
        sc.add_sphere(o2w, w2o, r, material=m, shape_id=j)
    sc.add_point_light(*light)
    sc.commit()
    my_rows = []
    for r in range(runs):
        pm, _ = sc.trace_photons(n, max_depth=30, rr_depth=3, seed=40 + r, flags=N.RT_RENDER_COMPAT)
        ph = pm.photons()
        my_rows.append(summary(ph["power"].astype(np.float64), ph["shape_id"]))
    R_, M_ = np.stack(ref_rows), np.stack(my_rows)
    se = np.sqrt(R_.var(0, ddof=1) / runs + M_.var(0, ddof=1) / runs)
    live = se > 0
    z = (M_.mean(0) - R_.mean(0))[live] / se[live]
    assert np.all(np.abs(z) < 4), z
    assert abs(M_[:, 0].mean() / R_[:, 0].mean() - 1) < 0.01  # stored photons per emitted photon
    # the glass sphere stores nothing (it is not a scattering material) on either side
    assert R_[:, 6].max() == 0 and M_[:, 6].max() == 0
