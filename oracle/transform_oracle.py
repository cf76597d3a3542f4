"""TEST INFRASTRUCTURE ONLY: CPU restatement of the second pass, local motions
-> one global transform per frame (vsLocalmotions2Transforms /
vsMotionsToTransform, src/localmotion2transform.c:40-330 of the reference),
for the similarity model and the rotational (fov) model.  The lens branch
(:59-105) is not restated.

The reference's shipped build compiles this code with -O3 -msse2 -ffast-math,
and its results depend on how that build groups and rounds a few
expressions.  Each of the following was pinned against the compiled reference
(oracle/_ref, through calcTransformQuality, mean, stddev and the whole
vsLocalmotions2Transforms) and is restated exactly here:

* mean (src/transformtype.c:401-409) is vectorised into two interleaved
  partial sums (even and odd elements), added together, then the odd tail;
  stddev (:421-428) is a plain sequential sum (its sqr() is an exported,
  interposable function that is not inlined, so the loop stays scalar);
* transform_vec_double (:193-209), similarity model: x' = (zcos*rx + zsin*ry)
  + (t.x + c_x), and likewise for y;
* prepare_transform_fov (:162-190): z = 1 + zoom*0.01 (the division by 100
  becomes a multiplication by its rounded reciprocal);
* calcTransformQuality (src/localmotion2transform.c:139-172): the error sum
  over the enabled fields is sequential in field order; the penalty is
  error/num + (|alpha|*0.2 + |zoom|*0.002), the two penalty terms added
  first;
* focal_from_fov (src/transformtype.c:123-127): (width/2) / tan(fov*(pi/360));
* the fov model's projection: X = (r0*rx + r1*ry) + r2*f (same for Y, Z),
  x' = ((z*f)*X)/Z + c_x;
* vsGradientDescent (src/localmotion2transform.c:288-330): the finite
  difference is a true division by h = +-1e-6.

Only tests/ and bench.py's CPU-baseline leg import this module.
"""
import math

import numpy as np

# vsMotionsToTransform's constants (src/localmotion2transform.c:242-250)
STEP_SIZES = (0.2, 0.2, 0.00005, 0.1)
GD_STEPS_PER_DIM = 16
GD_THRESHOLD = 0.01


def _seqsum(a):
    """left-to-right double sum (np.add.accumulate is a sequential scan)"""
    return float(np.add.accumulate(a)[-1]) if len(a) else 0.0


def ref_mean(a):
    """mean() as the reference build evaluates it: two interleaved partial sums"""
    n = len(a)
    n0 = n // 2 * 2
    s = _seqsum(a[0:n0:2]) + _seqsum(a[1:n0:2])
    for v in a[n0:]:
        s += float(v)
    return s / n


def ref_stddev(a, mu):
    d = a - mu
    return math.sqrt(_seqsum(d * d) / len(a))


def disable_fields(mask, quality, k):
    """disableFields, src/localmotion2transform.c:204-218 (mask updated in place)"""
    mu = ref_mean(quality)
    thresh = mu + k * ref_stddev(quality, mu)
    sel = quality > thresh
    mask[sel] = -1.0
    return int(sel.sum())


def wrap_angle(a):
    """new_transform's angle wrap, src/transformtype.c:38-58"""
    while a < -math.pi:
        a += 2.0 * math.pi
    while a > math.pi:
        a -= 2.0 * math.pi
    return a


def focal_from_fov(fov, width):
    if fov <= 0.0 or fov >= 180.0 or width <= 0:
        return 0.0
    return (width / 2.0) / math.tan(fov * (math.pi / 360.0))


def _mat3mul(a, b):
    t = [0.0] * 9
    for i in range(3):
        for j in range(3):
            s = 0.0
            for k in range(3):
                s += a[3 * i + k] * b[3 * k + j]
            t[3 * i + j] = s
    return t


def _rotation_forward(yaw, pitch, roll):
    """transpose of rotation_matrix_backward, src/transformtype.c:142-156,175-182"""
    cy, sy = math.cos(-yaw), math.sin(-yaw)
    cp, sp = math.cos(pitch), math.sin(pitch)
    cr, sr = math.cos(roll), math.sin(roll)
    ry = [cy, 0.0, sy, 0.0, 1.0, 0.0, -sy, 0.0, cy]
    rx = [1.0, 0.0, 0.0, 0.0, cp, -sp, 0.0, sp, cp]
    rz = [cr, -sr, 0.0, sr, cr, 0.0, 0.0, 0.0, 1.0]
    b = _mat3mul(_mat3mul(ry, rx), rz)
    return [b[0], b[3], b[6], b[1], b[4], b[7], b[2], b[5], b[8]]


class _Frame:
    def __init__(self, recs, width, height, fov):
        self.fx = recs["fx"].astype(np.float64)
        self.fy = recs["fy"].astype(np.float64)
        self.vx = recs["vx"].astype(np.float64)
        self.vy = recs["vy"].astype(np.float64)
        self.cx = float(width // 2)
        self.cy = float(height // 2)
        self.rx = self.fx - self.cx
        self.ry = self.fy - self.cy
        self.f = focal_from_fov(fov, width)


def transform_quality(p, fr, mm):
    """calcTransformQuality: writes the squared residual of every enabled field
    (mm >= 0) into mm and returns the penalised mean residual"""
    x, y, a, z = p
    a = wrap_angle(a)
    zz = 1.0 + z * 0.01
    if fr.f > 0.0:
        f = fr.f
        r = _rotation_forward(x / f, y / f, a)
        X = (r[0] * fr.rx + r[1] * fr.ry) + r[2] * f
        Y = (r[3] * fr.rx + r[4] * fr.ry) + r[5] * f
        Z = (r[6] * fr.rx + r[7] * fr.ry) + r[8] * f
        vx = ((zz * f) * X) / Z + fr.cx
        vy = ((zz * f) * Y) / Z + fr.cy
    else:
        zc, zs = zz * math.cos(a), zz * math.sin(a)
        vx = (zc * fr.rx + zs * fr.ry) + (x + fr.cx)
        vy = ((-zs) * fr.rx + zc * fr.ry) + (y + fr.cy)
    ex = (vx - fr.fx) - fr.vx
    ey = (vy - fr.fy) - fr.vy
    e = ex * ex + ey * ey
    en = mm >= 0
    mm[en] = e[en]
    num = 1 + int(en.sum())
    return _seqsum(e[en]) / num + (abs(a) * 0.2 + abs(z) * 0.002)


def gradient_descent(p, fr, mm, steps=GD_STEPS_PER_DIM, step_sizes=STEP_SIZES,
                     threshold=GD_THRESHOLD):
    """vsGradientDescent with calcTransformQuality as the objective"""
    dim = 4
    ss = list(step_sizes)
    x = [float(v) for v in p]
    v = transform_quality(x, fr, mm)
    i = 0
    while i < steps * dim and v > threshold:
        k = i % dim
        x2 = list(x)
        h = 1e-6 if (i // dim) % 2 else -1e-6
        x2[k] += h
        v2 = transform_quality(x2, fr, mm)
        g = (v - v2) / h
        x2 = [x[j] + ((g if j == k else 0.0) * ss[k]) for j in range(dim)]
        v2 = transform_quality(x2, fr, mm)
        if v2 < v:
            x, v = x2, v2
            ss[k] *= 1.2
        else:
            ss[k] /= 2.0
        i += 1
    return x, v


def motions_to_transform(recs, width, height, fov=0.0, smooth_zoom=0):
    """vsMotionsToTransform for one frame's LocalMotions (structured records
    with vx, vy, fx, fy, match).  Returns ((x, y, alpha, zoom, extra),
    residual, gradient-descent rounds)."""
    n = len(recs)
    if n == 0:
        return (0.0, 0.0, 0.0, 0.0, 1), None, 0
    fr = _Frame(recs, width, height, fov)
    params = [_seqsum(fr.vx) / n, _seqsum(fr.vy) / n, 0.0, 0.0]
    mm = np.zeros(n)
    disable_fields(mm, recs["match"].astype(np.float64).copy(), 1.5)
    for k in range(3):
        res, resid = gradient_descent(params, fr, mm)
        if (k == 0 and resid > 0.1) or (k == 1 and resid > 20):
            disable_fields(mm, mm.copy(), 1.0)
            params = res
        else:
            break
    x, y, a, z = res
    a = wrap_angle(a)
    extra = 1 if resid > 100 else 0
    if not smooth_zoom:
        z = 0.0
    return (x, y, a, z, extra), resid, k + 1


def motions_to_transforms(recs, first, width, height, fov=0.0, smooth_zoom=0):
    """vsLocalmotions2Transforms (lens estimate off) over a clip whose frame k
    holds recs[first[k]:first[k+1]]; returns an array of (x, y, alpha, zoom,
    extra) rows as float64 plus the per-frame residuals"""
    nf = len(first) - 1
    out = np.zeros((nf, 5))
    resid = np.full(nf, np.nan)
    for k in range(nf):
        t, r, _ = motions_to_transform(recs[first[k]:first[k + 1]], width, height, fov,
                                       smooth_zoom)
        out[k] = t
        if r is not None:
            resid[k] = r
    return out, resid
