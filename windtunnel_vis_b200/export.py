"""File formats for exported fields and series (src/analysis/export.ts:19-56).

vtk ... legacy-VTK binary (big-endian) STRUCTURED_POINTS file of a FieldExport, readable by
        ParaView / VisIt: velocity and mean velocity normalised by U, vorticity by U / L, Q by
        U^2 / L^2, Cp and mean Cp from the density (2 (rho - rhoRef) / (3 U^2)); coordinates in
        metres (cell size dx, points every stride cells, origin at the first cell centre)
csv ... comma-separated rows with '#' comment lines; numbers to 7 significant digits, non-finite
        values left empty
"""
import math

import numpy as np


def vtk(f: dict, dx: float, U: float, L: float, rho_ref: float, title: str) -> bytes:
    nx, ny, nz = f["dims"]
    n = nx * ny * nz
    h = dx * f["stride"]
    vel = np.asarray(f["vel"], np.float32).reshape(n, 4)
    mean = np.asarray(f["mean"], np.float32).reshape(n, 4)
    vort = np.asarray(f["vort"], np.float32).reshape(n, 4)
    parts = []

    def text(s):
        parts.append(s.encode())

    def floats(a):
        # per-value float32 from the JS-number (f64) expression, written big-endian
        parts.append(np.ascontiguousarray(a, dtype=">f4").tobytes())
        text("\n")

    fmt = js_number_string

    def cp(rho):
        return (2.0 * (rho.astype(np.float64) - rho_ref)) / (3.0 * U * U)

    text(f"# vtk DataFile Version 3.0\n{title[:250]}\nBINARY\nDATASET STRUCTURED_POINTS\n")
    text(f"DIMENSIONS {nx} {ny} {nz}\nORIGIN {fmt(0.5 * dx)} {fmt(0.5 * dx)} {fmt(0.5 * dx) if nz > 1 else 0}\n"
         f"SPACING {fmt(h)} {fmt(h)} {fmt(h)}\nPOINT_DATA {n}\n")
    text("VECTORS velocity float\n")
    floats(vel[:, :3].astype(np.float64) / U)
    text("VECTORS mean_velocity float\n")
    floats(mean[:, :3].astype(np.float64) / U)
    text("VECTORS vorticity float\n")
    floats(vort[:, :3].astype(np.float64) * L / U)
    text("SCALARS Cp float 1\nLOOKUP_TABLE default\n")
    floats(cp(vel[:, 3]))
    text("SCALARS mean_Cp float 1\nLOOKUP_TABLE default\n")
    floats(cp(mean[:, 3]))
    text("SCALARS Q_criterion float 1\nLOOKUP_TABLE default\n")
    floats(vort[:, 3].astype(np.float64) * L * L / (U * U))
    return b"".join(parts)


def js_number_string(x) -> str:
    """A JavaScript Number as String(x) prints it (ECMAScript Number::toString, radix 10): the
    shortest round-tripping digits, positional for 1e-7 <= |x| < 1e21, otherwise d.ddde+n."""
    x = float(x)
    if x != x:
        return "NaN"
    if x == 0:
        return "0"
    if math.isinf(x):
        return "Infinity" if x > 0 else "-Infinity"
    if x < 0:
        return "-" + js_number_string(-x)
    mant, _, exp = repr(x).partition("e")
    intpart, _, frac = mant.partition(".")
    digits = (intpart + frac).lstrip("0")
    # position of the decimal point relative to the first significant digit
    lead = len(intpart + frac) - len((intpart + frac).lstrip("0"))
    n = len(intpart) - lead + (int(exp) if exp else 0)
    digits = digits.rstrip("0") or "0"
    k = len(digits)
    if k <= n <= 21:
        return digits + "0" * (n - k)
    if 0 < n <= 21:
        return digits[:n] + "." + digits[n:]
    if -6 < n <= 0:
        return "0." + "0" * (-n) + digits
    e = n - 1
    return digits[0] + ("." + digits[1:] if k > 1 else "") + "e" + ("+" if e >= 0 else "-") + str(abs(e))


def _num(v):
    # export.ts:21: numbers as +v.toPrecision(7), non-finite values left empty
    if isinstance(v, str):
        return v
    if not math.isfinite(v):
        return ""
    return js_number_string(float(f"{v:.7g}"))


def csv(header, rows, comments=()) -> str:
    lines = [f"# {c}" for c in comments] + [",".join(header)]
    lines += [",".join(_num(v) for v in r) for r in rows]
    return "\n".join(lines) + "\n"
