"""Aerodynamic post-processing on the host (f64), the reference's analysis module.

coefficients ........ src/analysis/aero.ts:4-7
drag_newtons, Ema ... src/analysis/aero.ts:9-27
lattice_speed,
map_flow, format_re . src/analysis/units.ts:10-83  (lattice <-> SI mapping, watchdog multipliers)
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


AIR_RHO = 1.225  # kg / m^3
AIR_NU = 1.5e-5  # m^2 / s at 20 C
CS = 1.0 / math.sqrt(3.0)


def drag_newtons(cd, speed, area_m2):
    return 0.5 * AIR_RHO * speed * speed * cd * area_m2


class Ema:
    """Exponential moving average; non-finite samples are ignored."""

    def __init__(self, k):
        self.k = k
        self.value = math.nan

    def push(self, v):
        if not math.isfinite(v):
            return self.value
        self.value = v if math.isnan(self.value) else self.value + self.k * (v - self.value)
        return self.value

    def reset(self):
        self.value = math.nan


def lattice_speed(speed, v_max):
    """Lattice inlet speed for a real speed: 0.03 at rest to 0.08 at the top speed."""
    s = min(max(speed / v_max, 0.0), 1.0)
    return 0.03 + (0.08 - 0.03) * s


def map_flow(speed, length_m, nu_air, l_cells, v_max, nu_min, re_override=None, u_scale=1.0, nu_scale=1.0):
    """Real configuration -> lattice: the simulated Re is the real Re scaled so that the top speed
    reaches the grid's resolvable limit (0.08 L / nu_min); the watchdog multipliers lower U and
    raise nu. Returns {reReal, reSim, U, nu, tau, mach, dx, dt}."""
    re_real = speed * length_m / nu_air
    U = lattice_speed(speed, v_max) * u_scale
    re_max_grid = 0.08 * l_cells / nu_min
    re_real_max = v_max * length_m / AIR_NU
    re_sim = re_override if re_override and re_override > 0 else re_real * (re_max_grid / re_real_max)
    nu = U * l_cells / re_sim
    nu = max(nu * nu_scale, nu_min * 0.5)
    re_sim = U * l_cells / nu
    dx = length_m / l_cells
    dt = (U / speed) * dx if speed > 0 else 0.0
    return {"reReal": re_real, "reSim": re_sim, "U": U, "nu": nu, "tau": 3 * nu + 0.5, "mach": U / CS, "dx": dx,
            "dt": dt}


def format_re(re):
    if not math.isfinite(re):
        return "—"
    if re >= 1e6:
        return f"{re / 1e6:.2f}·10⁶"
    if re >= 1e4:
        return f"{re / 1e3:.0f}k"
    if re >= 1e3:
        return f"{re / 1e3:.1f}k"
    return f"{re:.0f}"


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
