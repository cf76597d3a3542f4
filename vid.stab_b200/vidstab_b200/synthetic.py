"""Seeded synthetic clips for tests and benchmarks.

No public dataset is involved: the clips are generated from a seed, with the
shapes and statistics of the benchmark configurations.

* a static "world" texture: 4-octave value noise mapped to luma [16, 235],
  plus Gaussian blobs and sharp-edged rectangles;
* a camera that walks over it (translation, rotation, zoom random walks);
* each frame is the world seen through the camera, bilinearly resampled,
  plus Gaussian sensor noise, rounded to uint8.

Warping uses torch (CPU or CUDA) when available for speed, else numpy.
"""
import math

import numpy as np


def value_noise(h, w, rng, octaves=4, base_cell=64):
    """Sum of `octaves` smoothly interpolated random grids, scaled to [0,1]."""
    out = np.zeros((h, w), np.float32)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cell = max(2, base_cell >> o)
        gh, gw = h // cell + 3, w // cell + 3
        grid = rng.random((gh, gw), dtype=np.float32)
        ys = np.arange(h, dtype=np.float32) / cell
        xs = np.arange(w, dtype=np.float32) / cell
        y0 = ys.astype(np.int64)
        x0 = xs.astype(np.int64)
        fy = ys - y0
        fx = xs - x0
        fy = fy * fy * (3 - 2 * fy)
        fx = fx * fx * (3 - 2 * fx)
        g00 = grid[y0][:, x0]
        g01 = grid[y0][:, x0 + 1]
        g10 = grid[y0 + 1][:, x0]
        g11 = grid[y0 + 1][:, x0 + 1]
        top = g00 + (g01 - g00) * fx[None, :]
        bot = g10 + (g11 - g10) * fx[None, :]
        out += amp * (top + (bot - top) * fy[:, None])
        total += amp
        amp *= 0.5
    out /= total
    lo, hi = out.min(), out.max()
    return (out - lo) / max(hi - lo, 1e-6)


def add_blobs(img, rng, n, smin=4.0, smax=40.0, amin=20.0, amax=80.0):
    h, w = img.shape
    for _ in range(n):
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        s = rng.uniform(smin, smax)
        a = rng.uniform(amin, amax) * (1 if rng.random() < 0.5 else -1)
        r = int(3 * s) + 1
        x0, x1 = max(0, int(cx) - r), min(w, int(cx) + r + 1)
        y0, y1 = max(0, int(cy) - r), min(h, int(cy) + r + 1)
        if x0 >= x1 or y0 >= y1:
            continue
        yy, xx = np.mgrid[y0:y1, x0:x1].astype(np.float32)
        img[y0:y1, x0:x1] += a * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * s * s))


def add_edges(img, rng, n, lmin=10, lmax=120, amin=15.0, amax=50.0):
    """sharp-edged rectangles (step edges in both directions)"""
    h, w = img.shape
    for _ in range(n):
        rw, rh = rng.integers(lmin, lmax), rng.integers(lmin, lmax)
        x0, y0 = rng.integers(0, max(1, w - rw)), rng.integers(0, max(1, h - rh))
        a = rng.uniform(amin, amax) * (1 if rng.random() < 0.5 else -1)
        img[y0:y0 + rh, x0:x0 + rw] += a


def world(h, w, seed, nblobs=200, edges=True, octaves=4):
    """Luma texture in [16,235] (float32)."""
    rng = np.random.default_rng(seed)
    img = 16.0 + 219.0 * value_noise(h, w, rng, octaves=octaves)
    add_blobs(img, rng, nblobs)
    if edges:
        add_edges(img, rng, nblobs // 2)
    return np.clip(img, 16.0, 235.0).astype(np.float32)


def _warp_numpy(src, coords_x, coords_y):
    h, w = src.shape
    x = np.clip(coords_x, 0, w - 1.001)
    y = np.clip(coords_y, 0, h - 1.001)
    x0 = x.astype(np.int64)
    y0 = y.astype(np.int64)
    fx = (x - x0).astype(np.float32)
    fy = (y - y0).astype(np.float32)
    a = src[y0, x0]
    b = src[y0, x0 + 1]
    c = src[y0 + 1, x0]
    d = src[y0 + 1, x0 + 1]
    top = a + (b - a) * fx
    bot = c + (d - c) * fx
    return top + (bot - top) * fy


def render(src, width, height, tx=0.0, ty=0.0, theta=0.0, zoom=1.0, center=None):
    """Frame (float32 H x W) of the camera at pose (tx, ty, theta, zoom): frame
    pixel p shows src at c_src + zoom * R(theta) (p - c_frame) + t."""
    hs, ws = src.shape
    cxs, cys = center if center is not None else ((ws - 1) / 2.0, (hs - 1) / 2.0)
    cxf, cyf = (width - 1) / 2.0, (height - 1) / 2.0
    ys, xs = np.mgrid[0:height, 0:width].astype(np.float32)
    rx, ry = xs - cxf, ys - cyf
    c, s = math.cos(theta), math.sin(theta)
    u = cxs + zoom * (c * rx - s * ry) + tx
    v = cys + zoom * (s * rx + c * ry) + ty
    return _warp_numpy(src, u, v)


def quantize(frame, rng, noise=2.0):
    f = frame
    if noise > 0:
        f = f + rng.normal(0.0, noise, size=f.shape).astype(np.float32)
    return np.clip(np.rint(f), 0, 255).astype(np.uint8)


def pair(width=640, height=480, seed=0, max_shift=8, max_rot_deg=1.0, noise=2.0, nblobs=20):
    """Frame A: value noise + blobs; frame B: A translated by an integer
    (dx,dy) in [-max_shift, max_shift], rotated by theta in +-max_rot_deg,
    bilinear, plus noise.  Returns (A, B, (dx, dy, theta))."""
    rng = np.random.default_rng(seed)
    A_f = world(height, width, seed, nblobs=nblobs, edges=False)
    A = np.clip(np.rint(A_f), 0, 255).astype(np.uint8)
    dx, dy = int(rng.integers(-max_shift, max_shift + 1)), int(rng.integers(-max_shift, max_shift + 1))
    theta = math.radians(rng.uniform(-max_rot_deg, max_rot_deg))
    # B(p) = A(R(-theta)(p - c - d) + c): content moves by d and rotates by theta
    h, w = A.shape
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float32)
    px, py = xs - cx - dx, ys - cy - dy
    c, s = math.cos(-theta), math.sin(-theta)
    u = cx + c * px - s * py
    v = cy + s * px + c * py
    B = quantize(_warp_numpy(A.astype(np.float32), u, v), rng, noise)
    return A, B, (dx, dy, theta)


def camera_path(nframes, seed, trans_sigma=3.0, rot_sigma_deg=0.2, zoom_sigma=0.002):
    """Random walk of (tx, ty, theta, zoom) per frame."""
    rng = np.random.default_rng(seed + 7919)
    steps = np.zeros((nframes, 4))
    steps[1:, 0:2] = rng.normal(0, trans_sigma, size=(nframes - 1, 2))
    steps[1:, 2] = np.radians(rng.normal(0, rot_sigma_deg, size=nframes - 1))
    steps[1:, 3] = rng.normal(0, zoom_sigma, size=nframes - 1)
    path = np.cumsum(steps, axis=0)
    path[:, 3] = np.exp(path[:, 3])  # multiplicative zoom
    return path


def clip(width, height, nframes, seed=1, trans_sigma=3.0, rot_sigma_deg=0.2, zoom_sigma=0.002,
         noise=2.0, nblobs=200, device=None, margin=None):
    """A camera-walk clip as uint8 (nframes, height, width).

    device=None: numpy on the CPU.  device="cuda"/"cpu": torch warping on that
    device, returns a torch uint8 tensor there (much faster for large clips)."""
    path = camera_path(nframes, seed, trans_sigma, rot_sigma_deg, zoom_sigma)
    H, W = _canvas(width, height, [path], margin)
    src = world(H, W, seed, nblobs=nblobs * max(1, (W * H) // (width * height)))
    return _render_clip(src, path, width, height, nframes, seed, noise, device)


def _canvas(width, height, paths, margin=None):
    """(H, W) of a world every camera path stays inside"""
    ext = max((np.abs(p[:, :2]).max() if len(p) > 1 else 0.0) for p in paths)
    rot = max((np.abs(p[:, 2]).max() if len(p) > 1 else 0.0) for p in paths)
    zmax = max(p[:, 3].max() for p in paths)
    diag = math.hypot(width, height) * max(1.0, zmax)
    if margin is None:
        margin = int(ext + (diag - min(width, height)) / 2 * (1 if rot > 0 else 0) + 32)
    W = int(max(width * zmax, diag if rot > 0 else width * zmax)) + 2 * margin
    H = int(max(height * zmax, diag if rot > 0 else height * zmax)) + 2 * margin
    return H, W


def clips_shared_world(width, height, nframes, seeds, world_seed, trans_sigma=3.0,
                       rot_sigma_deg=0.2, zoom_sigma=0.002, noise=2.0, nblobs=200, device=None):
    """One camera-walk clip per seed (its own path and sensor noise) over one
    shared scene generated from world_seed: many streams without generating
    a scene per stream."""
    paths = [camera_path(nframes, sd, trans_sigma, rot_sigma_deg, zoom_sigma) for sd in seeds]
    H, W = _canvas(width, height, paths)
    src = world(H, W, world_seed, nblobs=nblobs * max(1, (W * H) // (width * height)))
    return [_render_clip(src, p, width, height, nframes, sd, noise, device)
            for p, sd in zip(paths, seeds)]


def _render_clip(src, path, width, height, nframes, seed, noise, device):
    H, W = src.shape
    if device is None:
        rng = np.random.default_rng(seed + 31337)
        out = np.empty((nframes, height, width), np.uint8)
        for k in range(nframes):
            tx, ty, th, z = path[k]
            out[k] = quantize(render(src, width, height, tx, ty, th, z), rng, noise)
        return out
    import torch
    import torch.nn.functional as F
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 31337)
    srct = torch.from_numpy(src).to(dev)[None, None]
    ys, xs = torch.meshgrid(torch.arange(height, device=dev, dtype=torch.float32),
                            torch.arange(width, device=dev, dtype=torch.float32), indexing="ij")
    rx, ry = xs - (width - 1) / 2.0, ys - (height - 1) / 2.0
    cxs, cys = (W - 1) / 2.0, (H - 1) / 2.0
    out = torch.empty((nframes, height, width), dtype=torch.uint8, device=dev)
    for k in range(nframes):
        tx, ty, th, z = [float(v) for v in path[k]]
        c, s = math.cos(th), math.sin(th)
        u = cxs + z * (c * rx - s * ry) + tx
        v = cys + z * (s * rx + c * ry) + ty
        grid = torch.stack([u / (W - 1) * 2 - 1, v / (H - 1) * 2 - 1], dim=-1)[None]
        f = F.grid_sample(srct, grid, mode="bilinear", padding_mode="border", align_corners=True)[0, 0]
        if noise > 0:
            f = f + noise * torch.randn(f.shape, generator=g, device=dev)
        out[k] = f.round().clamp(0, 255).to(torch.uint8)
    return out


def to_packed(luma, bpp=3):
    """Interleaved RGB(A) frames with distinct but correlated channels."""
    y = luma.astype(np.int32)
    r = y
    g = np.clip((y * 7) // 8 + 20, 0, 255)
    b = np.clip(255 - y, 0, 255)
    chans = [r, g, b] + ([np.full_like(y, 255)] if bpp == 4 else [])
    st = np.stack(chans, axis=-1).astype(np.uint8)
    return st.reshape(*luma.shape[:-1], luma.shape[-1] * bpp)
