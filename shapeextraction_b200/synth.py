"""Seeded synthetic point clouds standing in for the reference's inputs.

The reference loads KITTI/OBJ/Semantic3D files (src/DataIO.cpp:13-121); no
dataset is available, so every workload is generated here from a seed with the
shapes, sizes and distributions of the benchmark configurations:

* ``uniform_cube``   100k points in U[0,1)^3 (30-bit codes, k=10 case)
* ``scene``          surfaces of 32 spheres (r in U[0.02, 0.2]) and 8 planes
                     clipped to the unit cube, area-weighted, Gaussian jitter
                     sigma=0.002 along the normal (2M points, k=16 case)
* ``precision_mix``  scene surfaces + anisotropic-noise planes + collinear
                     segments + 1e-4-scale clusters offset by 1e3
* ``gaussian_mixture`` 64 anisotropic Gaussians (density ratio up to 1000:1)
                     plus scene surfaces
* ``batched_clouds`` many independent scenes with log-uniform sizes

All generators return three contiguous float32 arrays (x, y, z) in a random
(shuffled) order, the SoA layout of PointCloud<float> (src/PointCloud.hpp:105-122).
"""
from __future__ import annotations

import numpy as np


def _unit(rng, n):
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v


def _plane_basis(nrm):
    a = np.array([1.0, 0.0, 0.0]) if abs(nrm[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    u = np.cross(nrm, a)
    u /= np.linalg.norm(u)
    v = np.cross(nrm, u)
    return u, v


_HALF = 1.75  # half-side of the in-plane square that covers the unit cube from any point inside it


def _sample_clipped_plane(rng, c, nrm, m, sigma):
    """m points uniform on the plane (c, nrm) clipped to [0,1]^3, jittered along nrm."""
    u, v = _plane_basis(nrm)
    out = np.empty((0, 3))
    while out.shape[0] < m:
        need = m - out.shape[0]
        ab = rng.uniform(-_HALF, _HALF, (max(4 * need, 1024), 2))
        p = c + ab[:, :1] * u + ab[:, 1:] * v
        inside = np.all((p >= 0.0) & (p <= 1.0), axis=1)
        out = np.concatenate([out, p[inside][:need]])
    if sigma > 0:
        out = out + rng.normal(0.0, sigma, (m, 1)) * nrm
    return out


def _plane_area(rng, c, nrm, samples=20000):
    u, v = _plane_basis(nrm)
    ab = rng.uniform(-_HALF, _HALF, (samples, 2))
    p = c + ab[:, :1] * u + ab[:, 1:] * v
    frac = np.mean(np.all((p >= 0.0) & (p <= 1.0), axis=1))
    return max(frac, 1e-3) * (2 * _HALF) ** 2


def _surface_points(rng, n, n_spheres=32, n_planes=8, sigma=0.002):
    radii = rng.uniform(0.02, 0.2, n_spheres)
    centers = rng.uniform(0.0, 1.0, (n_spheres, 3)) * (1.0 - 2.0 * radii[:, None]) + radii[:, None]
    pc = rng.uniform(0.2, 0.8, (n_planes, 3))
    pn = _unit(rng, n_planes)
    areas = np.concatenate([4.0 * np.pi * radii**2, [_plane_area(rng, pc[i], pn[i]) for i in range(n_planes)]])
    counts = rng.multinomial(n, areas / areas.sum())
    parts = []
    for i in range(n_spheres):
        m = counts[i]
        if m == 0:
            continue
        d = _unit(rng, m)
        r = radii[i] + (rng.normal(0.0, sigma, (m, 1)) if sigma > 0 else 0.0)
        parts.append(centers[i] + r * d)
    for j in range(n_planes):
        m = counts[n_spheres + j]
        if m:
            parts.append(_sample_clipped_plane(rng, pc[j], pn[j], m, sigma))
    return np.concatenate(parts) if parts else np.zeros((0, 3))


def _finish(rng, p):
    p = p[rng.permutation(p.shape[0])].astype(np.float32)
    return np.ascontiguousarray(p[:, 0]), np.ascontiguousarray(p[:, 1]), np.ascontiguousarray(p[:, 2])


def uniform_cube(n=100_000, seed=1):
    rng = np.random.default_rng(seed)
    return tuple(np.ascontiguousarray(rng.random(n, dtype=np.float32)) for _ in range(3))


def scene(n=2_000_000, seed=1, n_spheres=32, n_planes=8, sigma=0.002):
    rng = np.random.default_rng(seed)
    return _finish(rng, _surface_points(rng, n, n_spheres, n_planes, sigma))


def precision_mix(n=20_000_000, seed=1):
    """Well-conditioned surfaces mixed with near-degenerate neighbourhoods."""
    rng = np.random.default_rng(seed)
    n_surf = int(0.4 * n)
    n_aniso = int(0.25 * n)
    n_line = int(0.15 * n)
    n_clu = n - n_surf - n_aniso - n_line
    parts = [_surface_points(rng, n_surf)]
    # planes with anisotropic noise: sigma log-uniform in [1e-5, 1e-2]
    n_pl = 16
    cnt = rng.multinomial(n_aniso, np.full(n_pl, 1.0 / n_pl))
    for i in range(n_pl):
        sig = 10 ** rng.uniform(-5, -2)
        parts.append(_sample_clipped_plane(rng, rng.uniform(0.2, 0.8, 3), _unit(rng, 1)[0], cnt[i], sig))
    # collinear segments
    n_seg = 64
    cnt = rng.multinomial(n_line, np.full(n_seg, 1.0 / n_seg))
    for i in range(n_seg):
        a = rng.uniform(0, 1, 3)
        b = rng.uniform(0, 1, 3)
        t = rng.random((cnt[i], 1))
        parts.append(a + t * (b - a) + rng.normal(0, 1e-6, (cnt[i], 3)))
    # 1e-4-scale clusters offset by 1e3 from the origin
    n_c = 256
    cnt = rng.multinomial(n_clu, np.full(n_c, 1.0 / n_c))
    for i in range(n_c):
        c = 1e3 + rng.uniform(0, 1, 3)
        parts.append(c + rng.normal(0, 1e-4, (cnt[i], 3)))
    return _finish(rng, np.concatenate(parts))


def gaussian_mixture(n=50_000_000, seed=1, n_comp=64, surface_frac=0.25):
    """64 anisotropic Gaussians (density ratio up to 1000:1) plus scene surfaces."""
    rng = np.random.default_rng(seed)
    n_surf = int(surface_frac * n)
    n_g = n - n_surf
    # per-component density = weight / volume; spread weights and scales so the
    # densest component is ~1000x the sparsest
    w = 10 ** rng.uniform(0, 1.5, n_comp)
    cnt = rng.multinomial(n_g, w / w.sum())
    parts = [_surface_points(rng, n_surf)]
    for i in range(n_comp):
        scales = 10 ** rng.uniform(-2.2, -1.0, 3)
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        mu = rng.uniform(0.15, 0.85, 3)
        z = rng.standard_normal((cnt[i], 3)) * scales
        parts.append(mu + z @ q.T)
    return _finish(rng, np.concatenate(parts))


def batched_clouds(n_clouds=256, seed=1, lo=1_000, hi=500_000, ks=(8, 16, 32)):
    """Independent scenes with sizes exp(U[ln lo, ln hi]) and k drawn from ks."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), n_clouds)).astype(np.int64)
    kk = rng.choice(np.asarray(ks), n_clouds)
    clouds = [scene(int(sizes[i]), seed=seed * 100_003 + i) for i in range(n_clouds)]
    return clouds, kk


def tiny_cloud(n, seed=1):
    """Small random clouds for edge cases (duplicates likely on purpose)."""
    rng = np.random.default_rng(seed)
    p = rng.integers(0, 8, (n, 3)).astype(np.float32) / 7.0
    return _finish(rng, p)


def to_cloud_file(path, x, y, z):
    """Write the int64-n + SoA float32 file read by the reference driver."""
    with open(path, "wb") as f:
        np.asarray([x.size], np.int64).tofile(f)
        np.asarray(x, np.float32).tofile(f)
        np.asarray(y, np.float32).tofile(f)
        np.asarray(z, np.float32).tofile(f)
