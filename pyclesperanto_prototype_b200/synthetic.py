"""Seeded synthetic volumes with the shapes and value distributions of the
benchmark workloads (there is no public dataset for them):

  blobs_2d         2D float32 256x256: background N(10,3) clipped >= 0, 60
                   isotropic Gaussian blobs (sigma U(4,10) px, peak U(120,250))
                   at uniform centres, Poisson shot noise; seed 0.
  nuclei_volume    uint16 128x512x512 (z,y,x), 2:1:1 voxels: 2000
                   non-overlapping ellipsoids (semi-axes z U(3,6), y/x U(6,12)),
                   intensity U(800,3000) over background 100, Gaussian PSF
                   sigma (1.5,1,1), Poisson noise; seed 1.
  lightsheet_volume
                   uint16 512x1024x1024: 30000 ellipsoids (semi-axes U(4,10)),
                   dense enough that some touch, background 80..400 scaled by
                   a slow 3D sinusoid, Poisson noise; seed 2 (generated on the
                   GPU with torch; input generation is not part of any timed
                   region).
  blob_tile        a 2D or 3D tile of isotropic Gaussian blobs at a given
                   density per voxel, per-tile seed (batched / served forms).

Every generator takes its shape and object counts as arguments, so tests
build small instances with the same recipe.
"""
from __future__ import annotations

import math
import os

import numpy as np


def blobs_2d(shape=(256, 256), n_blobs=60, seed=0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    H, W = shape
    img = np.clip(rng.normal(10.0, 3.0, size=shape), 0, None)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    for _ in range(n_blobs):
        cy, cx = rng.uniform(0, H), rng.uniform(0, W)
        s = rng.uniform(4, 10)
        a = rng.uniform(120, 250)
        img += a * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s * s))
    img = rng.poisson(img).astype(np.float32)
    return img


def _ellipsoid_mask(az, ay, ax):
    rz, ry, rx = int(math.ceil(az)), int(math.ceil(ay)), int(math.ceil(ax))
    z, y, x = np.mgrid[-rz:rz + 1, -ry:ry + 1, -rx:rx + 1]
    return ((z / az) ** 2 + (y / ay) ** 2 + (x / ax) ** 2) <= 1.0


def nuclei_volume(shape=(128, 512, 512), n_objects=2000, seed=1, psf=(1.5, 1.0, 1.0),
                  background=100.0) -> np.ndarray:
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    D, H, W = shape
    vol = np.full(shape, background, np.float32)
    occ = np.zeros(shape, bool)
    placed = 0
    tries = 0
    while placed < n_objects and tries < n_objects * 20:
        tries += 1
        az, ay, ax = rng.uniform(3, 6), rng.uniform(6, 12), rng.uniform(6, 12)
        cz, cy, cx = int(rng.integers(0, D)), int(rng.integers(0, H)), int(rng.integers(0, W))
        inten = rng.uniform(800, 3000)
        m = _ellipsoid_mask(az, ay, ax)
        rz, ry, rx = (m.shape[0] // 2, m.shape[1] // 2, m.shape[2] // 2)
        z0, z1 = max(cz - rz, 0), min(cz + rz + 1, D)
        y0, y1 = max(cy - ry, 0), min(cy + ry + 1, H)
        x0, x1 = max(cx - rx, 0), min(cx + rx + 1, W)
        mm = m[z0 - (cz - rz):z1 - (cz - rz), y0 - (cy - ry):y1 - (cy - ry), x0 - (cx - rx):x1 - (cx - rx)]
        box = occ[z0:z1, y0:y1, x0:x1]
        if (box & mm).any():
            continue
        box |= mm
        vol[z0:z1, y0:y1, x0:x1][mm] = background + inten
        placed += 1
    vol = gaussian_filter(vol, sigma=psf)
    out = rng.poisson(vol)
    return np.clip(out, 0, 65535).astype(np.uint16)


def cached(name: str, fn, *args, **kwargs) -> np.ndarray:
    """Memoises a generated volume in $CLE_B200_CACHE (default /tmp)."""
    d = os.environ.get("CLE_B200_CACHE", "/tmp/cle_b200_cache")
    os.makedirs(d, exist_ok=True)
    p = os.path.join(d, name + ".npy")
    if os.path.exists(p):
        return np.load(p)
    a = fn(*args, **kwargs)
    np.save(p + ".tmp.npy", a)
    os.replace(p + ".tmp.npy", p)
    return a


def lightsheet_volume(shape=(512, 1024, 1024), n_objects=30000, seed=2, device="cuda"):
    """torch uint16 volume on `device`."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    D, H, W = shape
    z = torch.linspace(0, 1, D, device=device).view(D, 1, 1)
    y = torch.linspace(0, 1, H, device=device).view(1, H, 1)
    x = torch.linspace(0, 1, W, device=device).view(1, 1, W)
    bg = 240.0 + 160.0 * torch.sin(2 * math.pi * z + 1.0) * torch.cos(2 * math.pi * y) * torch.sin(
        math.pi * x + 0.5)
    vol = bg.expand(D, H, W).contiguous().to(torch.float32)
    prm = torch.rand((n_objects, 7), generator=g, device=device).cpu().numpy()
    for k in range(n_objects):
        cz, cy, cx = int(prm[k, 0] * D), int(prm[k, 1] * H), int(prm[k, 2] * W)
        az, ay, ax = 4 + 6 * prm[k, 3], 4 + 6 * prm[k, 4], 4 + 6 * prm[k, 5]
        inten = 800 + 2200 * prm[k, 6]
        rz, ry, rx = int(math.ceil(az)), int(math.ceil(ay)), int(math.ceil(ax))
        z0, z1 = max(cz - rz, 0), min(cz + rz + 1, D)
        y0, y1 = max(cy - ry, 0), min(cy + ry + 1, H)
        x0, x1 = max(cx - rx, 0), min(cx + rx + 1, W)
        zz = torch.arange(z0, z1, device=device, dtype=torch.float32).view(-1, 1, 1) - cz
        yy = torch.arange(y0, y1, device=device, dtype=torch.float32).view(1, -1, 1) - cy
        xx = torch.arange(x0, x1, device=device, dtype=torch.float32).view(1, 1, -1) - cx
        m = (zz / az) ** 2 + (yy / ay) ** 2 + (xx / ax) ** 2 <= 1.0
        sub = vol[z0:z1, y0:y1, x0:x1]
        sub[m] = float(inten)
    out = torch.poisson(vol, generator=g)
    return out.clamp_(0, 65535).to(torch.int32).to(torch.uint16)


def blob_tile(shape, density, seed, device="cuda"):
    """float32 torch tile: background N(10,3) clipped at 0, isotropic Gaussian
    blobs (sigma U(4,10), peak U(120,250)) at `density` blobs per voxel,
    Poisson noise.  Blobs are rendered per sigma class (1 px wide) by blurring
    impulses of weight peak / w0^d with the library's Gaussian (w0 = centre
    weight), so each blob has its drawn peak."""
    import torch
    from . import _ops
    from ._tier0 import B200Array

    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    shape = tuple(int(s) for s in shape)
    nvox = int(np.prod(shape))
    nb = max(1, int(round(density * nvox)))
    img = torch.clamp(10.0 + 3.0 * torch.randn(shape, generator=g, device=device), min=0.0)
    idx = torch.randint(0, nvox, (nb,), generator=g, device=device)
    sig = 4 + 6 * torch.rand(nb, generator=g, device=device)
    amp = 120 + 130 * torch.rand(nb, generator=g, device=device)
    cls = torch.clamp((sig - 4).floor().long(), 0, 5)
    for c in range(6):
        sel = cls == c
        if not bool(sel.any()):
            continue
        s_c = 4.5 + c
        n = int(8 * s_c) | 1
        r = n // 2
        w0 = 1.0 / float(np.exp(-(np.arange(-r, r + 1) ** 2) / (2 * s_c * s_c)).sum())
        imp = torch.zeros(nvox, device=device)
        imp.index_put_((idx[sel],), amp[sel] / (w0 ** len(shape)), accumulate=True)
        out = torch.empty(shape, dtype=torch.float32, device=device)
        _ops.gaussian_blur(B200Array(imp.view(shape)), B200Array(out), s_c, s_c, s_c)
        img += out
    return torch.poisson(img, generator=g).to(torch.float32)
