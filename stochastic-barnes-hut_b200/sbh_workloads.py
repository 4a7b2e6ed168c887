"""Seeded synthetic inputs for the summation workloads.

The reference publishes no benchmark data; its example drives the plugin with a
mesh sampled by third-party tools (python/example.py:18-47).  These generators
produce the workloads this library is measured on, all seeded numpy
``default_rng`` streams, all float32 like the reference's FLOAT:

* ``gaussian_mixture``: isotropic Gaussian clusters (plain-method workload);
* ``torus_surface``: area-uniform points on a torus with exact outward normals
  and equal area weights (winding-number workload);
* ``circle_points``: points on the unit circle with Gaussian jitter (2D smooth
  distance workload);
* ``sphere_surface``: uniform points on a sphere with outward normals (serving
  workload);
* ``uniform_queries``: queries uniform in a box;
* ``padded_box``: the points' bounding box grown by 0.01, as the reference's
  example does (python/example.py:23-24).
"""
from __future__ import annotations

import numpy as np


def padded_box(points: np.ndarray, pad: float = 0.01):
    lo = (points.min(axis=0) - pad).astype(np.float32)
    hi = (points.max(axis=0) + pad).astype(np.float32)
    return lo, hi


def gaussian_mixture(n: int, seed: int, dim: int = 3, clusters: int = 8, sigma: float = 0.05,
                     centre_range: float = 0.8, mass_range=(0.5, 1.5)):
    """Points from `clusters` equal-weight isotropic Gaussians with centres
    uniform in [-centre_range, centre_range]^dim; masses uniform in mass_range;
    unit normals uniform on the sphere."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-centre_range, centre_range, (clusters, dim))
    which = rng.integers(0, clusters, n)
    pts = centres[which] + rng.normal(0.0, sigma, (n, dim))
    nrm = rng.normal(size=(n, dim))
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-12)
    mass = rng.uniform(mass_range[0], mass_range[1], n)
    return pts.astype(np.float32), nrm.astype(np.float32), mass.astype(np.float32)


def torus_surface(n: int, seed: int, R: float = 0.6, r: float = 0.2, jitter: float = 0.0):
    """Area-uniform samples of the torus ((R + r cos v) cos u, (R + r cos v) sin u, r sin v):
    u uniform, v by rejection with acceptance (R + r cos v) / (R + r).  Normals are
    the exact outward normals; every point carries the area weight 4 pi^2 R r / n.
    Optional isotropic Gaussian jitter of standard deviation `jitter`."""
    rng = np.random.default_rng(seed)
    us, vs = [], []
    got = 0
    while got < n:
        m = int((n - got) * 1.4) + 1024
        u = rng.uniform(0.0, 2 * np.pi, m)
        v = rng.uniform(0.0, 2 * np.pi, m)
        keep = rng.uniform(0.0, 1.0, m) < (R + r * np.cos(v)) / (R + r)
        us.append(u[keep])
        vs.append(v[keep])
        got += int(keep.sum())
    u = np.concatenate(us)[:n]
    v = np.concatenate(vs)[:n]
    rad = R + r * np.cos(v)
    pts = np.stack([rad * np.cos(u), rad * np.sin(u), r * np.sin(v)], axis=1)
    nrm = np.stack([np.cos(v) * np.cos(u), np.cos(v) * np.sin(u), np.sin(v)], axis=1)
    if jitter > 0:
        pts = pts + rng.normal(0.0, jitter, pts.shape)
    area = np.full(n, 4 * np.pi ** 2 * R * r / n)
    return pts.astype(np.float32), nrm.astype(np.float32), area.astype(np.float32)


def sphere_surface(n: int, seed: int, radius: float = 0.8):
    """Uniform samples of a sphere with outward normals and area weights 4 pi r^2 / n."""
    rng = np.random.default_rng(seed)
    nrm = rng.normal(size=(n, 3))
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-12)
    area = np.full(n, 4 * np.pi * radius ** 2 / n)
    return (radius * nrm).astype(np.float32), nrm.astype(np.float32), area.astype(np.float32)


def circle_points(n: int, seed: int, jitter: float = 1e-3):
    """Unit-circle samples (uniform angle) with N(0, jitter^2) jitter; outward
    normals; unit masses."""
    rng = np.random.default_rng(seed)
    th = rng.uniform(0.0, 2 * np.pi, n)
    nrm = np.stack([np.cos(th), np.sin(th)], axis=1)
    pts = nrm + rng.normal(0.0, jitter, (n, 2))
    return pts.astype(np.float32), nrm.astype(np.float32), np.ones(n, np.float32)


def uniform_queries(n: int, seed: int, dim: int = 3, lo: float = -1.0, hi: float = 1.0):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, (n, dim)).astype(np.float32)


def samples_for_budget(budget: int, root_children: int) -> int:
    """Sampled paths per root child for a per-query budget of `budget` paths:
    the sampler draws samples_per_subdomain paths in every root child."""
    return max(1, int(round(budget / max(1, root_children))))
