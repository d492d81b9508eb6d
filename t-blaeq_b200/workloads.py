"""Seeded synthetic query workloads for the benchmark configurations.

All draws use numpy's PCG64 generator from a fixed seed. Centres are uniformly chosen data points
(decoded finest coordinates of the index itself), and widths / noise scale with each dimension's
extent, measured on a fixed sample of data points.

Configurations (sizes as in the benchmark definitions):
  small       N=500,000  D=5  ratios 80,40,20  seed 20260330  sigma divisor 2.2
              100 range boxes, half-width 5% of extent; 100 KNN points (+N(0,(1% extent)^2)), K=10
  batched     N=10,000,000  D=8  ratios 100,50,20  seed 1  sigma divisor 3.0
              4096 range boxes, half-widths log-uniform in [0.1%, 10%] of extent
  knn         N=50,000,000  D=16  ratios 100,50,20  seed 2  sigma divisor 2.5
              4096 KNN points (+N(0,(2% extent)^2)), half K=20 and half K=100
  serving     N=100,000,000  D=8  ratios 100,50,20  seed 3
"""
from __future__ import annotations

import numpy as np

CONFIGS = {
    "small": dict(N=500_000, D=5, ratios=(80, 40, 20), seed=20260330, sigma_divisor=2.2),
    "batched": dict(N=10_000_000, D=8, ratios=(100, 50, 20), seed=1, sigma_divisor=3.0),
    "knn": dict(N=50_000_000, D=16, ratios=(100, 50, 20), seed=2, sigma_divisor=2.5),
    "serving": dict(N=100_000_000, D=8, ratios=(100, 50, 20), seed=3, sigma_divisor=3.0),
}


def generate_index(handler_cls, name: str, **over):
    cfg = dict(CONFIGS[name])
    cfg.update(over)
    return handler_cls.generate(cfg["N"], cfg["D"], 1.0, 100.0, False, len(cfg["ratios"]) + 1, cfg["ratios"],
                                cfg["seed"], cfg["sigma_divisor"])


def extent(handler, sample: int = 65536, seed: int = 7):
    info = handler.info()
    rng = np.random.default_rng(seed)
    pos = rng.integers(0, info["N"], min(sample, info["N"]))
    pts, _ = handler.decode_points(pos)
    return pts.min(axis=0), pts.max(axis=0)


def range_boxes(handler, n: int, seed: int, half_width: float | None = None,
                log_uniform: tuple | None = None) -> np.ndarray:
    """n boxes (lo[D] | hi[D]) centred on uniformly chosen data points. Half-widths are either a
    fixed fraction of each dimension's extent or exp(U[ln a, ln b]) times the extent, per dimension."""
    info = handler.info()
    rng = np.random.default_rng(seed)
    lo_e, hi_e = extent(handler)
    ext = hi_e - lo_e
    centres, _ = handler.decode_points(rng.integers(0, info["N"], n))
    D = info["D"]
    if log_uniform is not None:
        a, b = log_uniform
        frac = np.exp(rng.uniform(np.log(a), np.log(b), (n, D)))
    else:
        frac = np.full((n, D), half_width if half_width is not None else 0.05)
    hw = frac * ext
    return np.ascontiguousarray(np.concatenate([centres - hw, centres + hw], axis=1))


def knn_points(handler, n: int, seed: int, noise: float) -> np.ndarray:
    info = handler.info()
    rng = np.random.default_rng(seed)
    lo_e, hi_e = extent(handler)
    ext = hi_e - lo_e
    centres, _ = handler.decode_points(rng.integers(0, info["N"], n))
    return np.ascontiguousarray(centres + rng.normal(0.0, 1.0, centres.shape) * (noise * ext))
