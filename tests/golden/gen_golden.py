"""Generates the golden fixtures in tests/golden/ from the reference renderer's OWN code
(oracle/_ref/libref_oracle.so, built from the reference sources by oracle/Makefile).

Run here, where the reference tree exists:  python tests/golden/gen_golden.py [--config1]
The fixtures are what the CPU tests check the C restatement against and what the GPU
tests check the CUDA path against, on machines where the reference tree is absent.
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from oracle import bindings  # noqa: E402
import cases  # noqa: E402

OUT = Path(__file__).resolve().parent


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def gen_small(R):
    out = {}
    for name, (v, f) in {
        "soup1000": cases.soup(1000, 11),
        "soup20000": cases.soup(20000, 12),
        "grids": cases.stacked_grids(),
    }.items():
        b = R.bvh(v, f)
        o, d = cases.edge_rays(5) if name == "grids" else __import__("importlib").import_module(
            "2023_render_engine_b200.scenes").random_rays(4096, seed=13, lo=-1.2, hi=1.2)
        ids = b.intersect(o, d)
        ids_sh = b.intersect(o, d, shadow=True)
        t = b.hit_t(ids, o, d)
        ex = b.export()
        out[name] = dict(v=v, f=f, o=o, d=d, ids=ids, t=t, sorted=ex["sorted"], codes=ex["codes"])
    np.savez_compressed(OUT / "trace_small.npz", **{f"{k}__{kk}": vv for k, d in out.items() for kk, vv in d.items()})
    # Cornell box spheres: the reference's matrices and sphere hits
    v, f, m, sph = cases.cornell_soup()
    rs = bindings.RefSpheres(R, [s["center"] for s in sph], [s["radius"] for s in sph], [s["glass"] for s in sph])
    S = __import__("importlib").import_module("2023_render_engine_b200.scenes")
    o, d = S.random_rays(4096, seed=21, lo=-1.0, hi=1.0)
    ids, t = rs.intersect(o, d)
    ids_sh, t_sh = rs.intersect(o, d, shadow=True)
    mats = {}
    for i in range(len(sph)):
        o2w, w2o = rs.matrices(i)
        mats[f"o2w{i}"], mats[f"w2o{i}"] = o2w, w2o
    np.savez_compressed(OUT / "spheres_cornell.npz", o=o, d=d, ids=ids, t=t, ids_shadow=ids_sh, t_shadow=t_sh,
                        centers=np.array([s["center"] for s in sph], np.float32),
                        radii=np.array([s["radius"] for s in sph], np.float32), **mats)
    # photon kd-tree k nearest (radius and shape filter)
    rng = np.random.default_rng(31)
    pos = rng.uniform(-1, 1, (20000, 3)).astype(np.float32)
    shp = rng.integers(0, 4, 20000).astype(np.int32)
    q = rng.uniform(-1, 1, (512, 3)).astype(np.float32)
    qs = rng.integers(-1, 4, 512).astype(np.int32)
    kd = bindings.RefKdTree(R, pos, shp)
    idx, cnt = kd.knn(q, 50, 0.25, qs)
    np.savez_compressed(OUT / "knn_small.npz", pos=pos, shape=shp, q=q, qshape=qs, k=50, radius=0.25, idx=idx,
                        count=cnt)


def gen_config1(R, nrays=1 << 24):
    S = __import__("importlib").import_module("2023_render_engine_b200.scenes")
    sc = S.stress_scene()
    v, f, m = S.flatten(sc)
    b = R.bvh(v, f)
    o, d = S.random_rays(nrays, seed=7)
    t0 = time.time()
    ids = b.intersect(o, d, threads=16)
    t1 = time.time()
    t = b.hit_t(ids, o, d, threads=16)
    info = {
        "scene": "stress_scene(subdiv=8, seed=1): displaced icosphere + Cornell box walls/light",
        "triangles": int(f.shape[0]),
        "vertices_sha256": sha(v),
        "indices_sha256": sha(f),
        "rays": nrays,
        "ray_seed": 7,
        "origins_sha256": sha(o),
        "directions_sha256": sha(d),
        "ids_sha256": sha(ids.astype(np.int32)),
        "t_sha256": sha(t.astype(np.float32)),
        "hit_fraction": float((ids >= 0).mean()),
        "reference_trace_seconds_16_threads": t1 - t0,
        "sample_index": list(range(0, nrays, nrays // 4096))[:4096],
    }
    info["sample_ids"] = ids[info["sample_index"]].tolist()
    (OUT / "config1_closest_hit.json").write_text(json.dumps(info, indent=1))


if __name__ == "__main__":
    R = bindings.RefOracle()
    gen_small(R)
    if "--config1" in sys.argv:
        gen_config1(R)
    print("golden fixtures written to", OUT)
