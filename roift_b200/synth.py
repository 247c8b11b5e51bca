"""Seeded synthetic volumes for the five OIFT + relaxation workloads.

The reference ships no datasets; every workload is generated here from a fixed
numpy PCG64 seed, so the CUDA path, the oracle and the reference CPU library see
the same bytes.  Shapes, intensities, noise, seeds and polarity follow the five
workload definitions (2D disc, 256^3 ellipsoid, 512x512x384 three-ellipsoid
pyramid case, 64-volume batch, 16 x 192^3 differentiation set).

Seed lists follow the reference CLI convention (oiftrelax.cpp:323-364): a flat list
of voxel addresses p = x + y*X + z*X*Y and a label per seed (0 = background).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Case:
    """One OIFT + relaxation job: an int16 (or uint8) volume, seeds, parameters."""

    name: str
    image: np.ndarray          # shape (Z, Y, X), int16 or uint8
    seeds: np.ndarray          # int32 voxel addresses
    seed_labels: np.ndarray    # int32 labels (0 = background)
    adjacency: int             # 4, 8, 6 or 26
    pol: float                 # polarity alpha in [-1, 1]
    sweeps: int                # relaxation sweeps
    weight_mode: str = "grad_q"  # "grad", "grad_q", "rbf_q", "blend_q"
    wq: int = 4095
    rbf_sigma: float = 150.0
    truth: np.ndarray | None = None  # ground-truth object mask (differentiation set)

    @property
    def shape(self):
        return self.image.shape

    @property
    def n(self):
        return int(self.image.size)

    def label_map(self) -> np.ndarray:
        """Label image with NIL (-1) everywhere except the seeds."""
        lab = np.full(self.n, -1, dtype=np.int32)
        lab[self.seeds] = self.seed_labels
        return lab


def _grid(Z, Y, X, dtype=np.float32):
    z = np.arange(Z, dtype=dtype)[:, None, None]
    y = np.arange(Y, dtype=dtype)[None, :, None]
    x = np.arange(X, dtype=dtype)[None, None, :]
    return z, y, x


def _boundary_seeds(shape, dist: int) -> np.ndarray:
    """Addresses of every voxel whose distance to the volume boundary is <= dist."""
    Z, Y, X = shape
    z, y, x = _grid(Z, Y, X, np.int32)
    d = np.minimum(np.minimum(np.minimum(x, X - 1 - x), np.minimum(y, Y - 1 - y)),
                   np.minimum(z, Z - 1 - z)) if Z > 1 else \
        np.minimum(np.minimum(x, X - 1 - x), np.minimum(y, Y - 1 - y))
    d = np.broadcast_to(d, shape)
    return np.flatnonzero(d.reshape(-1) <= dist).astype(np.int32)


def _sphere_seeds(shape, center, radius) -> np.ndarray:
    Z, Y, X = shape
    cz, cy, cx = center
    r = int(math.ceil(radius))
    zz, yy, xx = np.meshgrid(np.arange(max(0, int(cz) - r), min(Z, int(cz) + r + 2)),
                             np.arange(max(0, int(cy) - r), min(Y, int(cy) + r + 2)),
                             np.arange(max(0, int(cx) - r), min(X, int(cx) + r + 2)),
                             indexing="ij")
    m = (xx - cx) ** 2 + (yy - cy) ** 2 + (zz - cz) ** 2 <= radius * radius
    return (xx[m] + yy[m] * X + zz[m] * X * Y).astype(np.int32)


def _merge_seeds(groups):
    """Concatenate (addresses, label) groups; a voxel keeps its first label."""
    addr = np.concatenate([g[0] for g in groups]).astype(np.int32)
    lab = np.concatenate([np.full(len(g[0]), g[1], np.int32) for g in groups])
    _, first = np.unique(addr, return_index=True)
    first.sort()
    return addr[first], lab[first]


def disc2d(seed: int = 1, size: int = 256) -> Case:
    """2D 256x256 uint8 disc (r=70, 180 on 60, sigma 12), 4-adjacency, alpha +0.5,
    5x5 object seed block at the centre, 1-pixel border background, 10 sweeps."""
    rng = np.random.default_rng(seed)
    Y = X = size
    _, y, x = _grid(1, Y, X)
    c = (size - 1) / 2.0
    inside = (x - c) ** 2 + (y - c) ** 2 <= 70.0 ** 2
    img = np.where(inside, 180.0, 60.0) + rng.standard_normal((1, Y, X)) * 12.0
    img = np.clip(np.rint(img), 0, 255).astype(np.uint8)
    cx = size // 2
    blk = [(xx + yy * X) for yy in range(cx - 2, cx + 3) for xx in range(cx - 2, cx + 3)]
    obj = np.array(blk, np.int32)
    bg = _boundary_seeds((1, Y, X), 0)
    s, l = _merge_seeds([(obj, 1), (bg, 0)])
    return Case("disc2d_256", img, s, l, adjacency=4, pol=0.5, sweeps=10,
                weight_mode="grad")


def ellipsoid3d(seed: int = 2, size: int = 256, semi=(90, 70, 60), sweeps: int = 50,
                pol: float = -0.3) -> Case:
    """Config-2 volume: ellipsoid (90,70,60) at 1200 on 200, bias 1+0.1 sin(2 pi x/256),
    noise sigma 80, int16; seeds: sphere r=6 (object) and the distance<=2 boundary
    shell (background); 6-adjacency, uint16 [0,4095] gradient weights, alpha -0.3."""
    rng = np.random.default_rng(seed)
    Z = Y = X = size
    z, y, x = _grid(Z, Y, X)
    c = (size - 1) / 2.0
    s = size / 256.0
    a, b, cc = semi[0] * s, semi[1] * s, semi[2] * s
    inside = ((x - c) / a) ** 2 + ((y - c) / b) ** 2 + ((z - c) / cc) ** 2 <= 1.0
    img = np.where(inside, np.float32(1200.0), np.float32(200.0))
    img = img * (1.0 + 0.1 * np.sin(2.0 * np.pi * x / 256.0)).astype(np.float32)
    img = img + rng.standard_normal((Z, Y, X), dtype=np.float32) * np.float32(80.0)
    img = np.clip(np.rint(img), -32768, 32767).astype(np.int16)
    obj = _sphere_seeds((Z, Y, X), (c, c, c), 6.0 * max(s, 0.5))
    bg = _boundary_seeds((Z, Y, X), 2)
    sd, lb = _merge_seeds([(obj, 1), (bg, 0)])
    return Case(f"ellipsoid3d_{size}", img, sd, lb, adjacency=6, pol=pol, sweeps=sweeps,
                weight_mode="grad_q", wq=4095,
                truth=inside.reshape(Z, Y, X))


def three_ellipsoids(seed: int = 3, shape=(384, 512, 512), sweeps: int = 30) -> Case:
    """Config-3 volume: three overlapping ellipsoids {900,1100,1400} on 100, noise
    sigma 60, int16; 26-adjacency, RBF sigma 150 weights 4095(1-exp(-d^2/2s^2));
    three object spheres r=8 (labels 1..3) and a boundary background shell."""
    rng = np.random.default_rng(seed)
    Z, Y, X = shape
    z, y, x = _grid(Z, Y, X)
    sx, sy, sz = X / 512.0, Y / 512.0, Z / 384.0
    img = np.full((Z, Y, X), 100.0, np.float32)
    specs = [((0.40, 0.45, 0.50), (110, 90, 80), 900.0),
             ((0.58, 0.52, 0.48), (100, 120, 90), 1100.0),
             ((0.50, 0.62, 0.55), (70, 60, 70), 1400.0)]
    centers = []
    for (fx, fy, fz), (ax, ay, az), inten in specs:
        cx, cy, cz = fx * X, fy * Y, fz * Z
        centers.append((cz, cy, cx))
        m = (((x - cx) / (ax * sx)) ** 2 + ((y - cy) / (ay * sy)) ** 2
             + ((z - cz) / (az * sz)) ** 2) <= 1.0
        img = np.where(m, np.float32(inten), img)
    img = img + rng.standard_normal((Z, Y, X), dtype=np.float32) * np.float32(60.0)
    img = np.clip(np.rint(img), -32768, 32767).astype(np.int16)
    groups = []
    r = 8.0 * max(min(sx, sy, sz), 0.25)
    # object seeds at points of each ellipsoid that the later ones do not cover
    offs = [(-0.35, 0.0, 0.0), (0.30, 0.0, -0.3), (0.0, 0.0, 0.0)]
    for li, ((cz, cy, cx), (ox, oy, oz), (_, (ax, ay, az), _)) in enumerate(zip(centers, offs, specs)):
        c = (cz + oz * az * sz, cy + oy * ay * sy, cx + ox * ax * sx)
        groups.append((_sphere_seeds((Z, Y, X), c, r), li + 1))
    groups.append((_boundary_seeds((Z, Y, X), 1), 0))
    sd, lb = _merge_seeds(groups)
    return Case(f"three_ellipsoids_{X}x{Y}x{Z}", img, sd, lb, adjacency=26, pol=0.0,
                sweeps=sweeps, weight_mode="rbf_q", wq=4095, rbf_sigma=150.0)


def batch_mix(seed: int = 4, nvol: int = 64, sizes=(96, 128, 160, 192, 224, 256),
              sweeps: int = 20):
    """Config-4 batch: nvol volumes with per-axis sizes drawn from `sizes`, a random
    ellipsoid (semi-axes 0.2-0.4 of the extent, intensity U(600,1500)) on background
    U(50,300), noise sigma U(30,100); 2-8 seed sets per volume, each an object sphere
    r 4-8 at a random interior point plus the boundary shell; alpha U(-0.5,0.5).
    Returns a list of (Case, [seed sets]) where each seed set is (seeds, labels)."""
    rng = np.random.default_rng(seed)
    out = []
    for v in range(nvol):
        X, Y, Z = (int(rng.choice(sizes)) for _ in range(3))
        z, y, x = _grid(Z, Y, X)
        semi = rng.uniform(0.2, 0.4, 3) * np.array([X, Y, Z])
        ctr = np.array([X, Y, Z]) / 2.0 + rng.uniform(-0.1, 0.1, 3) * np.array([X, Y, Z])
        inside = (((x - ctr[0]) / semi[0]) ** 2 + ((y - ctr[1]) / semi[1]) ** 2
                  + ((z - ctr[2]) / semi[2]) ** 2) <= 1.0
        fg, bgv, sig = rng.uniform(600, 1500), rng.uniform(50, 300), rng.uniform(30, 100)
        img = np.where(inside, np.float32(fg), np.float32(bgv))
        img = img + rng.standard_normal((Z, Y, X), dtype=np.float32) * np.float32(sig)
        img = np.clip(np.rint(img), -32768, 32767).astype(np.int16)
        bg = _boundary_seeds((Z, Y, X), 1)
        sets = []
        for _ in range(int(rng.integers(2, 9))):
            r = float(rng.uniform(4, 8))
            # random interior point of the ellipsoid (radius fraction <= 0.5)
            u = rng.uniform(-0.5, 0.5, 3)
            pt = ctr + u * semi
            obj = _sphere_seeds((Z, Y, X), (pt[2], pt[1], pt[0]), r)
            sets.append(_merge_seeds([(obj, 1), (bg, 0)]))
        pol = float(rng.uniform(-0.5, 0.5))
        case = Case(f"batch{v}_{X}x{Y}x{Z}", img, sets[0][0], sets[0][1], adjacency=6,
                    pol=pol, sweeps=sweeps, weight_mode="grad_q", wq=4095)
        out.append((case, sets))
    return out


def diff_set(seed: int = 5, nvol: int = 16, size: int = 192):
    """Config-5 differentiation set: nvol ellipsoid volumes as in ellipsoid3d (scaled to
    `size`) with the ground-truth object mask."""
    return [ellipsoid3d(seed=seed * 1000 + i, size=size, sweeps=40) for i in range(nvol)]


def small_case(seed: int = 7, shape=(24, 20, 16), pol: float = -0.3, adjacency: int = 6,
               contrast: float = 1000.0, noise: float = 80.0, nlabels: int = 1,
               sweeps: int = 5, weight_mode: str = "grad") -> Case:
    """Small seeded case for parity tests: an ellipsoid (or nlabels blobs) in noise."""
    rng = np.random.default_rng(seed)
    Z, Y, X = shape
    z, y, x = _grid(Z, Y, X)
    img = np.full((Z, Y, X), 200.0, np.float32)
    groups = []
    for li in range(nlabels):
        cx = X * (0.5 if nlabels == 1 else 0.25 + 0.5 * li / max(nlabels - 1, 1))
        cy, cz = Y * 0.5, Z * 0.5
        ax, ay, az = X * 0.3 / max(1, nlabels ** 0.5), Y * 0.3, max(Z * 0.3, 0.5)
        m = ((x - cx) / ax) ** 2 + ((y - cy) / ay) ** 2 + (((z - cz) / az) ** 2 if Z > 1 else 0) <= 1.0
        img = np.where(m, np.float32(200.0 + contrast * (1 + 0.3 * li)), img)
        groups.append((_sphere_seeds((Z, Y, X), (cz if Z > 1 else 0, cy, cx),
                                     max(1.0, min(X, Y) * 0.06)), li + 1))
    img = img + rng.standard_normal((Z, Y, X), dtype=np.float32) * np.float32(noise)
    img = np.clip(np.rint(img), 0, 32767).astype(np.int16)
    groups.append((_boundary_seeds((Z, Y, X), 0), 0))
    sd, lb = _merge_seeds(groups)
    return Case(f"small_{X}x{Y}x{Z}", img, sd, lb, adjacency=adjacency, pol=pol,
                sweeps=sweeps, weight_mode=weight_mode)
