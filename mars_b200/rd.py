"""Rate-distortion comparison of two operating-point curves: BD-rate and BD-PSNR over
shape-preserving cubic (PCHIP) interpolation in the (log10 bpp, PSNR) plane, with the
preconditions of crates/mars-bench/src/bdrate.rs:49-81 (at least 4 points per curve, finite
positive points, strictly increasing in both bpp and PSNR) and its integration intervals
(bdrate.rs:141-204).  The interpolant is the Fritsch-Carlson PCHIP of
crates/mars-bench/src/pchip.rs (interior slopes by the weighted harmonic mean, the
three-point edge slope with its sign and 3x limits, Hermite basis integrated in closed
form).  Host-side measurement code: it is how the refinement mode's gain is quoted.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

MIN_POINTS_PER_CURVE = 4


class BdError(ValueError):
    """A curve pair that does not meet the BD contract (no number is produced)."""


def bpp(file_size_bytes: int, width: int, height: int) -> float:
    """metrics::bpp (crates/mars-core/src/metrics.rs:70-73)."""
    if width <= 0 or height <= 0:
        raise ValueError("bpp needs a non-empty image")
    return 8.0 * file_size_bytes / (width * height)


class Pchip:
    """Monotone piecewise-cubic Hermite interpolant through strictly increasing x."""

    def __init__(self, x, y):
        x, y = [float(v) for v in x], [float(v) for v in y]
        if len(x) != len(y):
            raise BdError(f"x and y must have equal length ({len(x)} vs {len(y)})")
        if len(x) < 2:
            raise BdError(f"need at least 2 points, got {len(x)}")
        for i in range(1, len(x)):
            if not x[i] > x[i - 1]:
                raise BdError(f"x values must be strictly increasing (violated at index {i})")
        n = len(x)
        h = [x[i + 1] - x[i] for i in range(n - 1)]
        delta = [(y[i + 1] - y[i]) / h[i] for i in range(n - 1)]
        d = [0.0] * n
        if n == 2:
            d[0] = d[1] = delta[0]
        else:
            for i in range(1, n - 1):
                if delta[i - 1] * delta[i] > 0.0:
                    w1 = 2.0 * h[i] + h[i - 1]
                    w2 = h[i] + 2.0 * h[i - 1]
                    d[i] = (w1 + w2) / (w1 / delta[i - 1] + w2 / delta[i])
            d[0] = _edge_slope(h[0], h[1], delta[0], delta[1])
            d[n - 1] = _edge_slope(h[n - 2], h[n - 3], delta[n - 2], delta[n - 3])
        self.x, self.y, self.d = x, y, d

    def _interval(self, t: float) -> int:
        n = len(self.x)
        lo, hi = 0, n
        while lo < hi:  # first index with x >= t
            mid = (lo + hi) // 2
            if self.x[mid] < t:
                lo = mid + 1
            else:
                hi = mid
        if lo < n and self.x[lo] == t:
            return min(lo, n - 2)
        return 0 if lo == 0 else min(lo - 1, n - 2)

    def eval(self, t: float) -> float:
        i = self._interval(t)
        h = self.x[i + 1] - self.x[i]
        s = (t - self.x[i]) / h
        s2, s3 = s * s, s * s * s
        return (self.y[i] * (2 * s3 - 3 * s2 + 1) + h * self.d[i] * (s3 - 2 * s2 + s)
                + self.y[i + 1] * (-2 * s3 + 3 * s2) + h * self.d[i + 1] * (s3 - s2))

    def integrate(self, a: float, b: float) -> float:
        lo, hi = self.x[0], self.x[-1]
        if a > b:
            raise BdError("integration bounds reversed")
        if a < lo - 1e-12 or b > hi + 1e-12:
            raise BdError(f"integration range [{a}, {b}] is outside [{lo}, {hi}]")
        a, b = max(a, lo), min(b, hi)
        total = 0.0
        for i in range(len(self.x) - 1):
            x0, x1 = self.x[i], self.x[i + 1]
            s_lo, s_hi = max(a, x0), min(b, x1)
            if s_hi <= s_lo:
                continue
            h = x1 - x0
            s0, s1 = (s_lo - x0) / h, (s_hi - x0) / h
            f00 = _a00(s1) - _a00(s0)
            f10 = _a10(s1) - _a10(s0)
            f01 = _a01(s1) - _a01(s0)
            f11 = _a11(s1) - _a11(s0)
            total += h * (self.y[i] * f00 + h * self.d[i] * f10 + self.y[i + 1] * f01
                          + h * self.d[i + 1] * f11)
        return total


def _sign(v: float) -> float:
    return math.copysign(1.0, v)


def _edge_slope(h0, h1, d0, d1):
    d = ((2.0 * h0 + h1) * d0 - h0 * d1) / (h0 + h1)
    if _sign(d) != _sign(d0):
        d = 0.0
    elif _sign(d0) != _sign(d1) and abs(d) > abs(3.0 * d0):
        d = 3.0 * d0
    return d


def _a00(s):
    return s ** 4 / 2.0 - s ** 3 + s


def _a10(s):
    return s ** 4 / 4.0 - 2.0 * s ** 3 / 3.0 + s * s / 2.0


def _a01(s):
    return -s ** 4 / 2.0 + s ** 3


def _a11(s):
    return s ** 4 / 4.0 - s ** 3 / 3.0


@dataclass
class BdResult:
    bd_rate_pct: float
    bd_psnr_db: float
    psnr_interval_db: tuple
    bpp_interval: tuple
    bd_psnr_bpp_interval: tuple
    points_reference: int
    points_test: int
    interpolation: str = "pchip(log10 bpp, psnr)"


def _prepared(label, points):
    if len(points) < MIN_POINTS_PER_CURVE:
        raise BdError(f"curve '{label}' has {len(points)} points; at least "
                      f"{MIN_POINTS_PER_CURVE} are required")
    for b, p in points:
        if not (b > 0.0) or not math.isfinite(p):
            raise BdError(f"curve '{label}' contains a non-finite or non-positive point "
                          f"(bpp={b}, psnr={p})")
    pts = sorted((float(b), float(p)) for b, p in points)
    for (b0, p0), (b1, p1) in zip(pts, pts[1:]):
        if not (b1 > b0) or not (p1 > p0):
            raise BdError(f"curve '{label}' is not monotonically increasing: "
                          f"{(b0, p0)} then {(b1, p1)}")
    return pts


def bd_metrics(reference, test, labels=("reference", "test")) -> BdResult:
    """BD-rate (%) and BD-PSNR (dB) of `test` against `reference`; each curve is a list of
    (bpp, psnr) points."""
    a, b = _prepared(labels[0], reference), _prepared(labels[1], test)
    ax, ay = [math.log10(p[0]) for p in a], [p[1] for p in a]
    bx, by = [math.log10(p[0]) for p in b], [p[1] for p in b]
    rate_a, rate_b = Pchip(ay, ax), Pchip(by, bx)
    y_lo, y_hi = max(ay[0], by[0]), min(ay[-1], by[-1])
    if not y_hi > y_lo:
        raise BdError(f"curves '{labels[0]}' and '{labels[1]}' have no overlapping PSNR range")
    span = y_hi - y_lo
    bd_rate = (10.0 ** ((rate_b.integrate(y_lo, y_hi) - rate_a.integrate(y_lo, y_hi)) / span)
               - 1.0) * 100.0
    ends = [rate_a.eval(y_lo), rate_b.eval(y_lo), rate_a.eval(y_hi), rate_b.eval(y_hi)]
    dist_a, dist_b = Pchip(ax, ay), Pchip(bx, by)
    x_lo, x_hi = max(ax[0], bx[0]), min(ax[-1], bx[-1])
    if not x_hi > x_lo:
        raise BdError(f"curves '{labels[0]}' and '{labels[1]}' have no overlapping bpp range")
    bd_psnr = (dist_b.integrate(x_lo, x_hi) - dist_a.integrate(x_lo, x_hi)) / (x_hi - x_lo)
    return BdResult(bd_rate, bd_psnr, (y_lo, y_hi), (10.0 ** min(ends), 10.0 ** max(ends)),
                    (10.0 ** x_lo, 10.0 ** x_hi), len(a), len(b))
