"""Seeded synthetic grayscale image pairs for ORB detect/describe/match workloads.

Image A is a sum of Gaussian blobs, overdrawn with filled rectangles and convex
polygons, plus Gaussian noise (sigma 3), clipped to [0, 255].  Image B is the
clean part of A warped by a random homography (rotation +-30 deg, scale
0.8-1.2, translation +-40 px, perspective terms +-1e-4) with fresh noise.

Everything is numpy with a fixed PCG64 seed per pair, so the same (seed, size)
gives the same bytes on every machine.  Images are returned as uint8 arrays
of shape (h, pitch) with pitch = align_up(w, 128) and zero padding, which is
the row layout the ORB entry points expect.
"""
import numpy as np

PAIR_SEED_BASE = 0x0B0000


def align_up(a, b):
    return (a + b - 1) // b * b


def _blobs(rng, img, n):
    h, w = img.shape
    cx = rng.uniform(0, w, n)
    cy = rng.uniform(0, h, n)
    sig = rng.uniform(2.0, 20.0, n)
    amp = rng.uniform(30.0, 200.0, n) * rng.choice([-1.0, 1.0], n)
    for i in range(n):
        r = int(np.ceil(3.0 * sig[i]))
        x0, x1 = max(0, int(cx[i]) - r), min(w, int(cx[i]) + r + 1)
        y0, y1 = max(0, int(cy[i]) - r), min(h, int(cy[i]) + r + 1)
        if x0 >= x1 or y0 >= y1:
            continue
        xs = np.arange(x0, x1, dtype=np.float64) - cx[i]
        ys = np.arange(y0, y1, dtype=np.float64) - cy[i]
        g = np.exp(-(ys[:, None] ** 2 + xs[None, :] ** 2) / (2.0 * sig[i] ** 2))
        img[y0:y1, x0:x1] += amp[i] * g


def _shapes(rng, img, n):
    h, w = img.shape
    m = min(w, h)
    for _ in range(n):
        val = rng.uniform(0.0, 255.0)
        if rng.uniform() < 0.5:
            rw = rng.uniform(0.02, 0.25) * w
            rh = rng.uniform(0.02, 0.25) * h
            x0 = rng.uniform(-0.1 * w, w)
            y0 = rng.uniform(-0.1 * h, h)
            xa, xb = int(max(0, x0)), int(min(w, x0 + rw))
            ya, yb = int(max(0, y0)), int(min(h, y0 + rh))
            if xa < xb and ya < yb:
                img[ya:yb, xa:xb] = val
        else:
            k = int(rng.integers(3, 9))
            cx = rng.uniform(0, w)
            cy = rng.uniform(0, h)
            rad = rng.uniform(0.02, 0.15) * m
            ang = np.sort(rng.uniform(0, 2 * np.pi, k))
            px = cx + rad * np.cos(ang)
            py = cy + rad * np.sin(ang)
            x0, x1 = max(0, int(np.floor(px.min()))), min(w, int(np.ceil(px.max())) + 1)
            y0, y1 = max(0, int(np.floor(py.min()))), min(h, int(np.ceil(py.max())) + 1)
            if x0 >= x1 or y0 >= y1:
                continue
            gx, gy = np.meshgrid(np.arange(x0, x1) + 0.5, np.arange(y0, y1) + 0.5)
            inside = np.ones(gx.shape, dtype=bool)
            for j in range(k):
                ax, ay = px[j], py[j]
                bx, by = px[(j + 1) % k], py[(j + 1) % k]
                # vertices are in counter-clockwise angular order: inside is left of each edge
                inside &= (bx - ax) * (gy - ay) - (by - ay) * (gx - ax) >= 0
            sub = img[y0:y1, x0:x1]
            sub[inside] = val


def _homography(rng, w, h):
    th = np.deg2rad(rng.uniform(-30.0, 30.0))
    s = rng.uniform(0.8, 1.2)
    tx, ty = rng.uniform(-40.0, 40.0, 2)
    p1, p2 = rng.uniform(-1e-4, 1e-4, 2)
    c, sn = np.cos(th), np.sin(th)
    cx, cy = w / 2.0, h / 2.0
    to_c = np.array([[1, 0, -cx], [0, 1, -cy], [0, 0, 1]], dtype=np.float64)
    from_c = np.array([[1, 0, cx + tx], [0, 1, cy + ty], [0, 0, 1]], dtype=np.float64)
    rs = np.array([[s * c, -s * sn, 0], [s * sn, s * c, 0], [p1, p2, 1]], dtype=np.float64)
    return from_c @ rs @ to_c


def _warp(img, H):
    """Bilinear inverse warp of img by homography H (dst = H * src); zeros outside."""
    h, w = img.shape
    Hi = np.linalg.inv(H)
    out = np.zeros_like(img)
    for y0 in range(0, h, 256):
        y1 = min(h, y0 + 256)
        gx, gy = np.meshgrid(np.arange(w, dtype=np.float64), np.arange(y0, y1, dtype=np.float64))
        den = Hi[2, 0] * gx + Hi[2, 1] * gy + Hi[2, 2]
        sx = (Hi[0, 0] * gx + Hi[0, 1] * gy + Hi[0, 2]) / den
        sy = (Hi[1, 0] * gx + Hi[1, 1] * gy + Hi[1, 2]) / den
        ix = np.floor(sx).astype(np.int64)
        iy = np.floor(sy).astype(np.int64)
        fx = sx - ix
        fy = sy - iy
        ok = (ix >= 0) & (iy >= 0) & (ix < w - 1) & (iy < h - 1)
        ixc = np.clip(ix, 0, w - 2)
        iyc = np.clip(iy, 0, h - 2)
        v = (img[iyc, ixc] * (1 - fx) * (1 - fy) + img[iyc, ixc + 1] * fx * (1 - fy)
             + img[iyc + 1, ixc] * (1 - fx) * fy + img[iyc + 1, ixc + 1] * fx * fy)
        out[y0:y1] = np.where(ok, v, 0.0)
    return out


def _finish(rng, clean, noise_sigma):
    noisy = clean + rng.standard_normal(clean.shape) * noise_sigma
    return np.clip(np.rint(noisy), 0, 255).astype(np.uint8)


def _pad(img8):
    h, w = img8.shape
    out = np.zeros((h, align_up(w, 128)), dtype=np.uint8)
    out[:, :w] = img8
    return out


def make_pair(w, h, seed=0, n_blobs=200, n_shapes=100, noise_sigma=3.0):
    """Return (A, B, H): two uint8 images of shape (h, align_up(w,128)) and the homography."""
    rng = np.random.Generator(np.random.PCG64(PAIR_SEED_BASE + int(seed)))
    r_img, r_noise_a, r_warp, r_noise_b = [np.random.Generator(np.random.PCG64(s))
                                            for s in rng.bit_generator.seed_seq.spawn(4)]
    clean = np.zeros((h, w), dtype=np.float64)
    _blobs(r_img, clean, n_blobs)
    _shapes(r_img, clean, n_shapes)
    a = _finish(r_noise_a, clean, noise_sigma)
    H = _homography(r_warp, w, h)
    b = _finish(r_noise_b, _warp(clean, H), noise_sigma)
    return _pad(a), _pad(b), H


def make_image(w, h, seed=0):
    """Image A of make_pair(w, h, seed) only (the warp is skipped)."""
    rng = np.random.Generator(np.random.PCG64(PAIR_SEED_BASE + int(seed)))
    r_img, r_noise_a, _, _ = [np.random.Generator(np.random.PCG64(s))
                              for s in rng.bit_generator.seed_seq.spawn(4)]
    clean = np.zeros((h, w), dtype=np.float64)
    _blobs(r_img, clean, 200)
    _shapes(r_img, clean, 100)
    return _pad(_finish(r_noise_a, clean, 3.0))


LEARNED_IMAGE_SEED = 0x100000  # images of the learned-proposal workload (disjoint from pair seeds)


def make_views(w, h, seed, views, n_blobs=200, n_shapes=100, noise_sigma=3.0):
    """Image A of make_pair(w, h, seed) and warped copies of its clean part, each
    with its own homography and noise.  views: a count n (views 0..n-1) or a list
    of view ids; view 0 is make_pair's B, view k >= 1 draws from its own pair of
    random streams, so a view is the same whichever other views are asked for."""
    ids = list(range(views)) if isinstance(views, int) else [int(v) for v in views]
    rng = np.random.Generator(np.random.PCG64(PAIR_SEED_BASE + int(seed)))
    ss = rng.bit_generator.seed_seq
    r_img, r_noise_a, r_warp, r_noise_b = [np.random.Generator(np.random.PCG64(s)) for s in ss.spawn(4)]
    top = max(ids) if ids else 0
    extra = ss.spawn(2 * max(0, top))
    clean = np.zeros((h, w), dtype=np.float64)
    _blobs(r_img, clean, n_blobs)
    _shapes(r_img, clean, n_shapes)
    a = _pad(_finish(r_noise_a, clean, noise_sigma))
    out = []
    for k in ids:
        if k == 0:
            rw, rn = r_warp, r_noise_b
        else:
            rw, rn = (np.random.Generator(np.random.PCG64(s)) for s in extra[2 * k - 2:2 * k])
        out.append(_pad(_finish(rn, _warp(clean, _homography(rw, w, h)), noise_sigma)))
    return a, out


def learned_image_set(args):
    """(index, view ids) -> (A, views) of the learned-proposal image with that
    index (1024 x 1024).  A top-level function so that a process pool can run it."""
    i, views = args
    return make_views(1024, 1024, LEARNED_IMAGE_SEED + int(i), list(views))


def random_descriptors(n, seed):
    """n uniform random 256-bit descriptors as uint8 (n, 32)."""
    rng = np.random.Generator(np.random.PCG64(0x0C0000 + int(seed)))
    return rng.integers(0, 256, size=(n, 32), dtype=np.uint8)


def match_workload(n_db, n_q, seed=0, flip_p=0.05):
    """Database of n_db uniform descriptors; n_q queries, the first half a copy of a
    random database row with each bit flipped with probability flip_p, the rest uniform."""
    rng = np.random.Generator(np.random.PCG64(0x0D0000 + int(seed)))
    db = rng.integers(0, 256, size=(n_db, 32), dtype=np.uint8)
    q = rng.integers(0, 256, size=(n_q, 32), dtype=np.uint8)
    half = n_q // 2
    src = rng.integers(0, n_db, size=half)
    bits = np.unpackbits(db[src], axis=1)
    flips = (rng.uniform(size=bits.shape) < flip_p).astype(np.uint8)
    q[:half] = np.packbits(bits ^ flips, axis=1)
    return db, q, src


# Resolutions of the batched workload (64 pairs of mixed size and keypoint cap).
BATCH_SIZES = [(320, 240), (640, 480), (1280, 720), (1920, 1080), (3840, 2160)]


def batch_layout(n_pairs=64, seed=0x0C3000):
    """(w, h, cap) per pair: resolutions uniform over BATCH_SIZES and keypoint
    caps uniform in [500, 10000]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = [BATCH_SIZES[int(i)] for i in rng.integers(0, len(BATCH_SIZES), n_pairs)]
    caps = [int(c) for c in rng.integers(500, 10001, n_pairs)]
    return [(w, h, c) for (w, h), c in zip(sizes, caps)]
