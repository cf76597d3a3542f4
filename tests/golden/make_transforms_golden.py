"""Generates tests/golden/transforms.npz: inputs and the unmodified
reference's outputs for the second pass (vsLocalmotions2Transforms,
src/localmotion2transform.c:40-121, lens estimate off).

Inputs: the reference detect's LocalMotions of two seeded synthetic clips
(640x480 x 12 frames, 1920x1080 x 8 frames) and hand-built record sets with
the edge cases of the fit (no motions, one, two, identical matches, a moving
object, motions no model fits, 825 fields of a 4K frame).  Outputs: the
reference's transforms for four configurations (fov 0 / 70 / 95 degrees,
smoothZoom 0 / 1).

Needs the reference build (make -C oracle REF=<reference checkout>):

    python tests/golden/make_transforms_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "vid.stab_b200"))

import oracle as O  # noqa: E402
from vidstab_b200 import synthetic as S  # noqa: E402

CONFIGS = ((0.0, 0), (0.0, 1), (70.0, 0), (95.0, 1))
TD = np.dtype([("x", "<f8"), ("y", "<f8"), ("alpha", "<f8"), ("zoom", "<f8"),
               ("barrel", "<f8"), ("rshutter", "<f8"), ("extra", "<i4"), ("pad", "<i4")])


def ref_transforms(recs, counts, width, height, fov, smooth_zoom):
    R = O.ref()
    R.vsref_motions_to_transforms.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                              C.c_double, C.c_int, C.c_int, C.c_void_p,
                                              C.c_void_p]
    first = np.zeros(len(counts) + 1, np.int64)
    first[1:] = np.cumsum(counts)
    out = np.zeros(len(counts), TD)
    el = C.c_double()
    rc = R.vsref_motions_to_transforms(width, height, recs.ctypes.data if len(recs) else None,
                                       first.ctypes.data, len(counts), fov, smooth_zoom, 0,
                                       out.ctypes.data, C.byref(el))
    assert rc == 0
    return np.stack([out["x"], out["y"], out["alpha"], out["zoom"],
                     out["extra"].astype(np.float64)], 1)


def grid_fields(width, height, size, step):
    xs = np.arange(size, width - size, step)
    ys = np.arange(size, height - size, step)
    gx, gy = np.meshgrid(xs, ys)
    return gx.ravel().astype(np.int16), gy.ravel().astype(np.int16)


def model_motions(fx, fy, width, height, tx, ty, alpha, zoom, rng, noise=0.6):
    cx, cy = width // 2, height // 2
    z = 1.0 + zoom / 100.0
    rx, ry = fx - cx, fy - cy
    px = z * np.cos(alpha) * rx + z * np.sin(alpha) * ry + tx + cx
    py = -z * np.sin(alpha) * rx + z * np.cos(alpha) * ry + ty + cy
    vx = np.rint(px - fx + rng.normal(0, noise, len(fx)))
    vy = np.rint(py - fy + rng.normal(0, noise, len(fy)))
    return vx.astype(np.int16), vy.astype(np.int16)


def records(vx, vy, fx, fy, size, match, contrast=0.3):
    r = np.zeros(len(vx), O.LM_DTYPE)
    r["vx"], r["vy"], r["fx"], r["fy"] = vx, vy, fx, fy
    r["fsize"] = size
    r["match"] = match
    r["contrast"] = contrast
    return r


def edge_sets(rng):
    """(name, records) of one 1920x1080 frame each"""
    W, H = 1920, 1080
    sets = [("empty", np.zeros(0, O.LM_DTYPE))]
    sets.append(("one", records([3], [-2], [900], [500], 32, [4.0])))
    sets.append(("two", records([3, 4], [-2, -1], [400, 1500], [300, 800], 32, [4.0, 6.0])))
    fx, fy = grid_fields(W, H, 112, 160)
    sets.append(("translation_equal_match",
                 records(np.full(len(fx), 5), np.full(len(fx), -7), fx, fy, 112,
                         np.full(len(fx), 3.5))))
    fx, fy = grid_fields(W, H, 32, 64)
    vx, vy = model_motions(fx, fy, W, H, 4.2, -3.1, 0.004, 0.3, rng)
    obj = (fx > 1200) & (fx < 1500) & (fy > 300) & (fy < 700)
    vx[obj] += 25
    vy[obj] -= 18
    match = rng.gamma(3.0, 2.0, len(fx))
    match[obj] *= 0.8
    sets.append(("moving_object", records(vx, vy, fx, fy, 32, match)))
    vx = rng.integers(-60, 60, len(fx)).astype(np.int16)
    vy = rng.integers(-60, 60, len(fx)).astype(np.int16)
    sets.append(("no_model", records(vx, vy, fx, fy, 32, rng.gamma(3.0, 2.0, len(fx)))))
    W4, H4 = 3840, 2160
    fx, fy = grid_fields(W4, H4, 48, 96)
    fx, fy = fx[:825], fy[:825]
    vx, vy = model_motions(fx, fy, W4, H4, -11.0, 6.5, -0.005, -0.5, rng)
    sets.append(("4k_825", records(vx, vy, fx, fy, 48, rng.gamma(3.0, 2.0, len(fx)))))
    return sets


def main():
    out = {}
    for name, (W, H, N, seed) in (("clip640", (640, 480, 12, 3)), ("clip1080", (1920, 1080, 8, 5))):
        frames = np.asarray(S.clip(W, H, N, seed=seed))
        recs, counts, _ = O.ref_clip(frames)
        out[name + "_recs"] = recs
        out[name + "_counts"] = counts.astype(np.int64)
        out[name + "_geom"] = np.array([W, H])
        for ci, (fov, sz) in enumerate(CONFIGS):
            out["%s_ref%d" % (name, ci)] = ref_transforms(recs, counts, W, H, fov, sz)
    rng = np.random.default_rng(17)
    sets = edge_sets(rng)
    for si, (name, r) in enumerate(sets):
        W, H = (3840, 2160) if name.startswith("4k") else (1920, 1080)
        out["edge%d_recs" % si] = r
        out["edge%d_geom" % si] = np.array([W, H])
        for ci, (fov, sz) in enumerate(CONFIGS):
            out["edge%d_ref%d" % (si, ci)] = ref_transforms(r, [len(r)], W, H, fov, sz)
    out["edge_names"] = np.array([n for n, _ in sets])
    out["configs"] = np.array(CONFIGS, np.float64)
    np.savez_compressed(os.path.join(HERE, "transforms.npz"), **out)
    print("wrote", os.path.join(HERE, "transforms.npz"))


if __name__ == "__main__":
    main()
