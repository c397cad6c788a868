"""Fitting (volume_scale, contrast_density) against experimental SAXS data.

Restatement of the reference's fit module (src/fit.rs), the consumer that runs
on top of the cached Debye model: experimental data (:19-135), the natural
cubic spline onto experimental q (:143-190), the analytic scale and χ²/N
(:194-234), box-clamped Nelder–Mead (:263-327) and the exhaustive grid fit
(:446-517). Each cost evaluation is one O(nq) recombination of the six
cached terms — no pair sum is recomputed.
"""
from __future__ import annotations

import bisect
import logging
from dataclasses import dataclass
from typing import Callable, Sequence, Tuple

import numpy as np

from .errors import InternalError, ValidationError

log = logging.getLogger(__name__)

DEFAULT_C1_BOUNDS = (0.5, 2.0)   # src/fit.rs:253
DEFAULT_C2_BOUNDS = (0.0, 0.1)   # src/fit.rs:259


@dataclass
class ExpData:
    q: list
    intensity: list
    sigma: list

    @classmethod
    def from_arrays(cls, q, intensity, sigma=()) -> "ExpData":
        q = [float(x) for x in q]
        intensity = [float(x) for x in intensity]
        sigma = [float(x) for x in sigma] if sigma is not None else []
        if not q:
            raise ValidationError("experimental data is empty")
        if len(intensity) != len(q):
            raise ValidationError(f"q ({len(q)}) and intensity ({len(intensity)}) length mismatch")
        if not sigma:
            sigma = [1.0] * len(q)
        elif len(sigma) != len(q):
            raise ValidationError(f"q ({len(q)}) and sigma ({len(sigma)}) length mismatch")
        return cls(q, intensity, sigma)

    @classmethod
    def from_file(cls, path) -> "ExpData":
        """CSV or whitespace columns q, I [, σ]; comment, alphabetic and blank
        lines skipped (src/fit.rs:31-103)."""
        q, inten, sig = [], [], []
        with open(path, "r", encoding="utf-8") as fh:
            for line in fh:
                t = line.strip()
                if not t or t.startswith("#") or t[0].isalpha():
                    continue
                parts = [p.strip() for p in t.split(",")] if "," in t else t.split()
                if len(parts) < 2:
                    continue
                try:
                    qi, ii = float(parts[0]), float(parts[1])
                except ValueError:
                    continue
                try:
                    si = float(parts[2]) if len(parts) > 2 else 1.0
                except ValueError:
                    si = 1.0
                q.append(qi)
                inten.append(ii)
                sig.append(si)
        if not q:
            raise ValidationError(f"no data points found in {path}")
        return cls(q, inten, sig)

    def q_max(self) -> float:
        return max([0.0] + self.q)


class CubicSpline:
    """Natural cubic spline (Numerical Recipes §3.3), src/fit.rs:143-190."""

    def __init__(self, xs: Sequence[float], ys: Sequence[float]):
        self.xs = [float(x) for x in xs]
        self.ys = [float(y) for y in ys]
        n = len(self.xs)
        self.y2 = [0.0] * n
        if n < 3:
            return
        xs, ys, y2 = self.xs, self.ys, self.y2
        u = [0.0] * n
        for i in range(1, n - 1):
            sig = (xs[i] - xs[i - 1]) / (xs[i + 1] - xs[i - 1])
            p = sig * y2[i - 1] + 2.0
            y2[i] = (sig - 1.0) / p
            u[i] = (ys[i + 1] - ys[i]) / (xs[i + 1] - xs[i]) - (ys[i] - ys[i - 1]) / (xs[i] - xs[i - 1])
            u[i] = (6.0 * u[i] / (xs[i + 1] - xs[i - 1]) - sig * u[i - 1]) / p
        for i in range(n - 2, -1, -1):
            y2[i] = y2[i] * y2[i + 1] + u[i]

    def eval(self, x: float) -> float:
        xs, ys = self.xs, self.ys
        if x <= xs[0]:
            return ys[0]
        if x >= xs[-1]:
            return ys[-1]
        i = bisect.bisect_left(xs, x)  # partition_point(v < x)
        if i == 0:
            return ys[0]
        x0, x1 = xs[i - 1], xs[i]
        y0, y1 = ys[i - 1], ys[i]
        d0, d1 = self.y2[i - 1], self.y2[i]
        h = x1 - x0
        a = (x1 - x) / h
        b = (x - x0) / h
        return a * y0 + b * y1 + ((a * a * a - a) * d0 + (b * b * b - b) * d1) * h * h / 6.0


def compute_scale(theory, exp: ExpData) -> float:
    """Σ(I_th·I_exp/σ²) / Σ(I_th²/σ²) (src/fit.rs:194-205)."""
    sp = CubicSpline(theory.q, theory.total)
    num = den = 0.0
    for q, ie, s in zip(exp.q, exp.intensity, exp.sigma):
        it = sp.eval(q)
        s2 = s * s
        num += it * ie / s2
        den += it * it / s2
    return num / den


def chi2_per_point(theory, exp: ExpData) -> float:
    """χ²/N with the analytic scale (src/fit.rs:209-234)."""
    n = float(len(exp.q))
    sp = CubicSpline(theory.q, theory.total)
    interp = [sp.eval(q) for q in exp.q]
    num = den = 0.0
    for it, ie, s in zip(interp, exp.intensity, exp.sigma):
        s2 = s * s
        num += it * ie / s2
        den += it * it / s2
    scale = num / den
    chi2 = 0.0
    for it, ie, s in zip(interp, exp.intensity, exp.sigma):
        r = (scale * it - ie) / s
        chi2 += r * r
    return chi2 / n


@dataclass
class FitResult:
    volume_scale: float
    contrast_density: float
    chi2: float
    scale: float


def _validate_bounds(name, b):
    lo, hi = b
    if not (np.isfinite(lo) and np.isfinite(hi)) or lo > hi:
        raise ValidationError(f"{name} bounds must be finite with lo <= hi (got {b})")


def _clamp(x, lo, hi):
    return min(max(x, lo), hi)


def nelder_mead_2d(cost, initial, c1b, c2b):
    """Box-clamped Nelder–Mead, ≤500 iterations, tolerance 1e-10
    (src/fit.rs:263-327)."""
    def ev(x, y):
        cx, cy = _clamp(x, *c1b), _clamp(y, *c2b)
        return (cx, cy, cost(cx, cy))

    simplex = [ev(x, y) for x, y in initial]
    for _ in range(500):
        simplex.sort(key=lambda t: t[2])
        if simplex[2][2] - simplex[0][2] < 1e-10:
            break
        cx = 0.5 * (simplex[0][0] + simplex[1][0])
        cy = 0.5 * (simplex[0][1] + simplex[1][1])
        rx, ry, fr = ev(2.0 * cx - simplex[2][0], 2.0 * cy - simplex[2][1])
        if fr < simplex[0][2]:
            ex, ey, fe = ev(3.0 * cx - 2.0 * simplex[2][0], 3.0 * cy - 2.0 * simplex[2][1])
            simplex[2] = (ex, ey, fe) if fe < fr else (rx, ry, fr)
        elif fr < simplex[1][2]:
            simplex[2] = (rx, ry, fr)
        else:
            kx, ky, fk = ev(0.5 * (cx + simplex[2][0]), 0.5 * (cy + simplex[2][1]))
            if fk < simplex[2][2]:
                simplex[2] = (kx, ky, fk)
            else:
                for i in (1, 2):
                    simplex[i] = ev(0.5 * (simplex[i][0] + simplex[0][0]),
                                    0.5 * (simplex[i][1] + simplex[0][1]))
    simplex.sort(key=lambda t: t[2])
    return simplex[0]


def _bounded_offset(start, bounds, preferred):
    delta = min(abs(preferred), (bounds[1] - bounds[0]) / 2.0)
    if preferred >= 0.0:
        return start + delta if start + delta <= bounds[1] else start - delta
    return start - delta if start - delta >= bounds[0] else start + delta


def _initial_simplex(c1b, c2b):
    c1 = _clamp(1.0, *c1b)
    c2 = _clamp(0.03, *c2b)
    return [(c1, c2), (_bounded_offset(c1, c1b, 0.08), c2), (c1, _bounded_offset(c2, c2b, -0.015))]


def fit_parameters_with_bounds(exp: ExpData, eval_fn: Callable, c1b=DEFAULT_C1_BOUNDS,
                               c2b=DEFAULT_C2_BOUNDS) -> FitResult:
    """src/fit.rs:365-411"""
    _validate_bounds("c1", c1b)
    _validate_bounds("c2", c2b)
    cost = lambda c1, c2: chi2_per_point(eval_fn(c1, c2), exp)
    c1, c2, chi2 = nelder_mead_2d(cost, _initial_simplex(c1b, c2b), c1b, c2b)
    scale = compute_scale(eval_fn(c1, c2), exp)
    return FitResult(c1, c2, chi2, scale)


def fit_parameters(exp: ExpData, eval_fn: Callable) -> FitResult:
    return fit_parameters_with_bounds(exp, eval_fn)


def fit_parameters_grid_with_bounds(exp: ExpData, eval_fn: Callable, c1_points: int,
                                    c2_points: int, c1b=DEFAULT_C1_BOUNDS,
                                    c2b=DEFAULT_C2_BOUNDS) -> FitResult:
    """Endpoint-inclusive exhaustive grid (src/fit.rs:446-517)."""
    if c1_points < 2 or c2_points < 2:
        raise ValidationError(
            f"grid fit requires at least 2 points per axis (got c1_points={c1_points}, "
            f"c2_points={c2_points})")
    _validate_bounds("c1", c1b)
    _validate_bounds("c2", c2b)
    gv = lambda b, n, i: b[0] + (b[1] - b[0]) * i / (n - 1)
    best = None
    for i in range(c1_points):
        c1 = gv(c1b, c1_points, i)
        for j in range(c2_points):
            c2 = gv(c2b, c2_points, j)
            chi2 = chi2_per_point(eval_fn(c1, c2), exp)
            if not np.isfinite(chi2):
                continue
            if best is None or chi2 < best[2]:
                best = (c1, c2, chi2)
    if best is None:
        raise InternalError("grid fit did not find any finite χ² value")
    c1, c2, chi2 = best
    return FitResult(c1, c2, chi2, compute_scale(eval_fn(c1, c2), exp))
