"""Seeded synthetic inputs for the Debye workloads.

Public SAXS datasets are not available offline, so every workload runs on
synthetic structures with the shapes and value distributions of the
benchmark configurations:

  globule      N atoms by random sequential addition (RSA) with a 1.2 Å
               minimum spacing, in a sphere or a prolate ellipsoid; species
               C/N/O/S drawn 0.63/0.17/0.19/0.01.
  exposure     atoms within 3 Å of the envelope surface are exposed with
               probability 0.35; an exposed atom gets the fully-exposed SASA
               shell weight 4π(r_s + 1.8)²·3/30 of its species radius r_s
               (src/solvent/sasa.rs:54-59 with area = the full sphere).
  trajectory   per-frame Gaussian displacements of a base structure, frame
               weights Dirichlet(1) (normalised Exp(1) draws).
  stream       Poisson arrivals of globules with log-uniform atom counts.

The RSA inserts candidates in batches against a cell grid whose cells hold at
most one atom (edge 1.2/√3 Å); a candidate is rejected if any accepted atom,
or an earlier candidate of its batch, lies within 1.2 Å. The minimum spacing
is therefore exact; relative to one-at-a-time RSA a batch may reject a few
extra candidates, which only changes which random points are kept.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

ELEMENTS = ("C", "N", "O", "S")
ELEMENT_PROBS = (0.63, 0.17, 0.19, 0.01)
D_MIN = 1.2
SURFACE_SHELL = 3.0
EXPOSED_PROB = 0.35
PROBE = 1.8


def _inside(p: np.ndarray, axes: np.ndarray) -> np.ndarray:
    return np.sum((p / axes) ** 2, axis=1) <= 1.0


def rsa_points(n: int, axes, rng: np.random.Generator, d_min: float = D_MIN) -> np.ndarray:
    """n points inside the ellipsoid with semi-axes `axes` (a sphere if equal),
    pairwise at least d_min apart, by batched RSA on a cell grid."""
    axes = np.asarray(axes, dtype=np.float64).reshape(3)
    h = d_min / math.sqrt(3.0)
    dims = np.ceil(2.0 * axes / h).astype(np.int64) + 5
    grid = np.full(int(np.prod(dims)), -1, dtype=np.int64)
    origin = -axes - 2.0 * h
    pts = np.empty((n, 3), dtype=np.float64)
    count = 0
    offs = np.array([(i, j, k) for i in range(-2, 3) for j in range(-2, 3) for k in range(-2, 3)
                     if (i, j, k) != (0, 0, 0)], dtype=np.int64)
    strides = np.array([dims[1] * dims[2], dims[2], 1], dtype=np.int64)
    stall = 0
    while count < n:
        need = n - count
        b = int(min(max(2 * need, 1024), 200_000))
        cand = rng.uniform(-1.0, 1.0, size=(b, 3)) * axes
        cand = cand[_inside(cand, axes)]
        if len(cand) == 0:
            continue
        cell3 = np.floor((cand - origin) / h).astype(np.int64)
        cid = cell3 @ strides
        ok = grid[cid] < 0
        cand, cell3, cid = cand[ok], cell3[ok], cid[ok]
        # one candidate per cell: keep the earliest
        _, first = np.unique(cid, return_index=True)
        first.sort()
        cand, cell3, cid = cand[first], cell3[first], cid[first]
        m = len(cand)
        if m == 0:
            stall += 1
            if stall > 1000:
                raise RuntimeError("RSA stalled: the requested density is too high")
            continue
        tmp_ids = count + np.arange(m, dtype=np.int64)
        # Scratch copy of the candidate coordinates addressed by id.
        allp = np.concatenate([pts[:count], cand])
        grid[cid] = tmp_ids
        reject = np.zeros(m, dtype=bool)
        for o in offs:
            nid = grid[(cell3 + o) @ strides]
            has = nid >= 0
            # existing atoms, or earlier candidates of this batch
            earlier = has & (nid < tmp_ids)
            if not earlier.any():
                continue
            d2 = np.sum((allp[np.where(earlier, nid, 0)] - cand) ** 2, axis=1)
            reject |= earlier & (d2 < d_min * d_min)
        keep = ~reject
        take = np.nonzero(keep)[0][:need]
        keep_mask = np.zeros(m, dtype=bool)
        keep_mask[take] = True
        grid[cid[~keep_mask]] = -1
        # re-number kept candidates contiguously after `count`
        k = len(take)
        grid[cid[take]] = count + np.arange(k, dtype=np.int64)
        pts[count:count + k] = cand[take]
        count += k
    return pts


def surface_distance(p: np.ndarray, axes) -> np.ndarray:
    """Distance from interior points to the ellipsoid surface. The closest
    surface point is x_i = a_i² p_i / (t + a_i²) for the root t in
    (-min a², 0] of Σ (a_i p_i / (t + a_i²))² = 1; the root is bracketed and
    found by bisection (monotone function), vectorised over points."""
    a = np.asarray(axes, dtype=np.float64).reshape(1, 3)
    a2 = a * a
    if np.allclose(a, a[0, 0]):
        return a[0, 0] - np.linalg.norm(p, axis=1)
    # A zero coordinate on a shorter axis puts the root at the pole t = -a²
    # (closest points off that axis); a 1e-6 Å nudge moves it inside the
    # bracket at a distance error of ~1e-6 Å.
    p = np.where(p == 0.0, 1e-6, p)
    lo = np.full(len(p), -a2.min() * (1.0 - 1e-15))
    hi = np.zeros(len(p))
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        f = np.sum((a * p / (mid[:, None] + a2)) ** 2, axis=1) - 1.0
        big = f > 0.0
        lo = np.where(big, mid, lo)
        hi = np.where(big, hi, mid)
    t = 0.5 * (lo + hi)
    x = a2 * p / (t[:, None] + a2)
    return np.linalg.norm(p - x, axis=1)


@dataclass
class Globule:
    pos: np.ndarray          # [N, 3] Å
    elements: np.ndarray     # [N] index into ELEMENTS
    exposed: np.ndarray      # [N] bool
    axes: Tuple[float, float, float]


def globule(n: int, axes, seed: int) -> Globule:
    """RSA globule with species and surface exposure flags."""
    rng = np.random.default_rng(seed)
    axes = tuple(float(a) for a in (axes if np.ndim(axes) else (axes, axes, axes)))
    pos = rsa_points(n, axes, rng)
    elements = rng.choice(len(ELEMENTS), size=n, p=ELEMENT_PROBS).astype(np.int64)
    near = surface_distance(pos, axes) <= SURFACE_SHELL
    exposed = near & (rng.random(n) < EXPOSED_PROB)
    return Globule(pos, elements, exposed, axes)


def sphere_radius_for(n: int) -> float:
    """Radius keeping the 1,000-atom / 16 Å density: R = 16·(N/1000)^{1/3}."""
    return 16.0 * (n / 1000.0) ** (1.0 / 3.0)


def trajectory(base: np.ndarray, n_frames: int, sigma: float, seed: int):
    """Frames [F, N, 3] = base + N(0, σ²) per coordinate, and Dirichlet(1)
    frame weights."""
    rng = np.random.default_rng(seed)
    frames = base[None, :, :] + rng.normal(0.0, sigma, size=(n_frames,) + base.shape)
    e = rng.exponential(1.0, size=n_frames)
    return frames, e / e.sum()


@dataclass
class StreamRequest:
    arrival: float           # s after the stream start
    n_atoms: int
    nq: int
    qmax: float
    solvent: bool
    seed: int


def request_stream(n_requests: int, rate_hz: float, seed: int, n_min: int = 500,
                   n_max: int = 50_000) -> List[StreamRequest]:
    """Poisson arrivals; N log-uniform in [n_min, n_max], nq uniform in
    100..1000, qmax uniform in [0.3, 1.0], solvent with probability 0.7."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, size=n_requests))
    ns = np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=n_requests)).astype(np.int64)
    nqs = rng.integers(100, 1001, size=n_requests)
    qmaxs = rng.uniform(0.3, 1.0, size=n_requests)
    solv = rng.random(n_requests) < 0.7
    seeds = rng.integers(0, 2**31 - 1, size=n_requests)
    return [StreamRequest(float(t[i]), int(ns[i]), int(nqs[i]), float(qmaxs[i]), bool(solv[i]),
                          int(seeds[i])) for i in range(n_requests)]
