"""Aerodynamic post-processing on the host (f64), the reference's analysis module.

coefficients ........ src/analysis/aero.ts:4-7
window_stats ........ src/analysis/aero.ts:33-52  (batch means, 8 batches)
crossing_frequency .. src/analysis/strouhal.ts:5-30
sphere_cd_ref ....... src/analysis/strouhal.ts:33-35  (Schiller-Naumann)
cylinder_st_ref ..... src/analysis/strouhal.ts:38-40  (Williamson fit)
"""
import math


def coefficients(fx, fy, fz, U, area, rho=1.0):
    """C = F / (1/2 rho U^2 A); in 2-D `area` is the frontal height in cells."""
    q = 0.5 * rho * U * U * max(area, 1e-9)
    return {"cd": fx / q, "cl": fy / q, "cs": fz / q}


def window_stats(t, v, window):
    """Mean and standard error of a correlated signal over its last `window` time units by the
    method of batch means (8 contiguous batches)."""
    n = len(t)
    if n < 16:
        return {"mean": math.nan, "se": math.nan, "span": 0.0, "n": n}
    t_end = t[n - 1]
    i0 = n - 1
    while i0 > 0 and t[i0 - 1] >= t_end - window:
        i0 -= 1
    span = t_end - t[i0]
    B = 8
    sums = [0.0] * B
    cnt = [0] * B
    tot = 0.0
    tot_n = 0
    for i in range(i0, n):
        b = min(B - 1, math.floor(((t[i] - t[i0]) / max(span, 1e-9)) * B))
        sums[b] += v[i]
        cnt[b] += 1
        tot += v[i]
        tot_n += 1
    mean = tot / tot_n
    bm = [s / c for s, c in zip(sums, cnt) if c]
    bm = [x for x in bm if math.isfinite(x)]
    if len(bm) < 4:
        return {"mean": mean, "se": math.nan, "span": span, "n": tot_n}
    var_b = sum((x - mean) ** 2 for x in bm) / (len(bm) - 1)
    return {"mean": mean, "se": math.sqrt(var_b / len(bm)), "span": span, "n": tot_n}


def crossing_frequency(t, v):
    """Dominant frequency from upward mean crossings with 15 % hysteresis; NaN with fewer than
    4 upward crossings (3 full cycles)."""
    n = len(v)
    if n < 8:
        return {"f": math.nan, "cycles": 0, "amplitude": math.nan}
    mean = sum(v) / n
    lo, hi = min(v), max(v)
    amp = (hi - lo) / 2
    hyst = amp * 0.15
    ups = []
    armed = v[0] < mean - hyst
    for i in range(1, n):
        if v[i] < mean - hyst:
            armed = True
        if armed and v[i - 1] < mean and v[i] >= mean:
            a = (mean - v[i - 1]) / (v[i] - v[i - 1])
            ups.append(t[i - 1] + a * (t[i] - t[i - 1]))
            armed = False
    if len(ups) < 4:
        return {"f": math.nan, "cycles": max(0, len(ups) - 1), "amplitude": amp}
    cycles = len(ups) - 1
    period = (ups[-1] - ups[0]) / cycles
    return {"f": 1.0 / period, "cycles": cycles, "amplitude": amp}


def sphere_cd_ref(re):
    return (24.0 / re) * (1.0 + 0.15 * re ** 0.687)


def cylinder_st_ref(re):
    return 0.2175 - 5.106 / re
