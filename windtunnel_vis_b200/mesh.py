"""Host-side mesh preparation for the voxelizer (f64 numpy).

normalize_mesh ...... src/voxelize/mesh.ts:271-318  (length 1 along +x, ground at y = 0, centred)
placement_matrix .... src/voxelize/mesh.ts:354-379  (column-major 4x4 mesh -> grid matrix)
grid_wheels ......... src/voxelize/mesh.ts:321-333  (wheels into grid space)
signed_volume ....... src/voxelize/mesh.ts:62-71

Geometry generators (our own, seeded; the reference builds its presets with three.js, which is
not part of this path):
uv_sphere ........... latitude/longitude sphere with the segment counts of the reference's sphere
                      preset (96 x 64), used by the voxelizer acceptance check
vehicle_body ........ superellipsoid body (length : width : height = 4 : 1.5 : 1.2) with four
                      16-segment cylinder wheels of radius 0.12 * height, ~200k triangles
"""
import math

import numpy as np


# ---- 4x4 matrices, column-major like three.js Matrix4.elements --------------------------------
def _mat(rows):
    return np.array(rows, np.float64)


def rot_y(a):
    c, s = math.cos(a), math.sin(a)
    return _mat([[c, 0, s, 0], [0, 1, 0, 0], [-s, 0, c, 0], [0, 0, 0, 1]])


def rot_z(a):
    c, s = math.cos(a), math.sin(a)
    return _mat([[c, -s, 0, 0], [s, c, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]])


def rot_x(a):
    c, s = math.cos(a), math.sin(a)
    return _mat([[1, 0, 0, 0], [0, c, -s, 0], [0, s, c, 0], [0, 0, 0, 1]])


def scale(sx, sy, sz):
    return np.diag([sx, sy, sz, 1.0])


def translate(x, y, z):
    m = np.eye(4)
    m[:3, 3] = [x, y, z]
    return m


def elements(m):
    """Row-major 4x4 -> column-major 16 (Matrix4.elements order)."""
    return np.asarray(m, np.float64).T.ravel().copy()


def apply(m, pts):
    p = np.asarray(pts, np.float64).reshape(-1, 3)
    return p @ m[:3, :3].T + m[:3, 3]


# ---- mesh helpers ------------------------------------------------------------------------------
def signed_volume(pos, idx):
    p = np.asarray(pos, np.float64).reshape(-1, 3)
    t = np.asarray(idx, np.int64).reshape(-1, 3)
    a, b, c = p[t[:, 0]], p[t[:, 1]], p[t[:, 2]]
    return float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)


def orient_outward(pos, idx):
    idx = np.asarray(idx, np.uint32).reshape(-1, 3)
    if signed_volume(pos, idx) < 0:
        idx = idx[:, [0, 2, 1]]
    return np.ascontiguousarray(idx.ravel())


def normalize_mesh(pos, align_longest=True, up="y", flip=False):
    """Returns (positions f32, min, max, transform 4x4): longest horizontal extent on +x, length
    1, centred in x and z, lowest point on y = 0."""
    p = np.asarray(pos, np.float64).reshape(-1, 3)
    total = np.eye(4)

    def app(m):
        nonlocal p, total
        total = m @ total
        p = apply(m, p)

    if up == "z":
        app(rot_x(-math.pi / 2))
    if align_longest:
        sx = p[:, 0].max() - p[:, 0].min()
        sz = p[:, 2].max() - p[:, 2].min()
        if sz > sx * 1.05:
            app(rot_y(math.pi / 2))
    if flip:
        app(rot_y(math.pi))
    lo, hi = p.min(0), p.max(0)
    ln = max(hi[0] - lo[0], 1e-9)
    cx, cz = (hi[0] + lo[0]) / 2, (hi[2] + lo[2]) / 2
    app(scale(1 / ln, 1 / ln, 1 / ln) @ translate(-cx, -lo[1], -cz))
    return p.astype(np.float32), p.min(0), p.max(0), total


def placement_matrix(positions, mesh_min, mesh_max, dims, pl):
    """placementMatrix: pl = {mode: 'ground'|'center', lengthFrac, diamFrac, xFrac, yawDeg,
    pitchDeg, rideCells, spanwise}. Returns (column-major 16 f64, scale, row-major 4x4)."""
    nx, ny, nz = dims
    height = mesh_max[1] - mesh_min[1]
    s = pl["lengthFrac"] * nx if pl["mode"] == "ground" else (pl["diamFrac"] * ny) / max(height, 1e-6)
    cy = (mesh_max[1] + mesh_min[1]) / 2
    R = rot_y(pl.get("yawDeg", 0) * math.pi / 180) @ rot_z(-pl.get("pitchDeg", 0) * math.pi / 180)
    if pl.get("spanwise"):
        sz = (nz + 4) / max(mesh_max[2] - mesh_min[2], 1e-6) if nz > 1 else s
    else:
        sz = s
    S = scale(s, s, sz)
    Cm = translate(0, -cy, 0)
    M = R @ S @ Cm
    p = np.asarray(positions, np.float64).reshape(-1, 3)
    stride = max(1, (p.shape[0] // 200000))
    min_y = apply(M, p[::stride])[:, 1].min()
    zc = nz / 2 if nz > 1 else 0.5
    ty = -min_y + pl.get("rideCells", 0) if pl["mode"] == "ground" else ny / 2 + 0.37
    T = translate(pl.get("xFrac", 0.35) * nx, ty, zc)
    full = T @ M
    return elements(full), s, full


def grid_wheels(wheels, m_rowmajor):
    """Wheels (normalized space) -> grid space: centre through M, axis through the linear part
    (normalised; half-width scaled by its length), radius by the x scale of M."""
    lin = m_rowmajor[:3, :3]
    sx = np.linalg.norm(lin[:, 0]) * (1 if np.linalg.det(lin) >= 0 else -1)
    out = []
    for w in wheels:
        c = apply(m_rowmajor, np.asarray(w["c"], np.float64))[0]
        a = lin @ np.asarray(w["axis"], np.float64)
        al = np.linalg.norm(a)
        out.append({"c": c.tolist(), "axis": (a / al).tolist(), "r": w["r"] * sx, "hw": w["hw"] * al})
    return out


# ---- generators --------------------------------------------------------------------------------
def uv_sphere(radius=0.5, w_seg=96, h_seg=64):
    """Latitude/longitude sphere: (w_seg + 1) x (h_seg + 1) vertex grid, pole rows without the
    degenerate triangles, outward-oriented. Returns (positions f32 (n,3), indices u32)."""
    v = np.arange(h_seg + 1) / h_seg
    u = np.arange(w_seg + 1) / w_seg
    th = v[:, None] * math.pi
    ph = u[None, :] * 2 * math.pi
    x = -radius * np.cos(ph) * np.sin(th)
    y = radius * np.cos(th) * np.ones_like(ph)
    z = radius * np.sin(ph) * np.sin(th)
    pos = np.stack([x, y, z], -1).reshape(-1, 3)
    g = np.arange((h_seg + 1) * (w_seg + 1)).reshape(h_seg + 1, w_seg + 1)
    tris = []
    for iy in range(h_seg):
        for ix in range(w_seg):
            a, b, c, d = g[iy, ix + 1], g[iy, ix], g[iy + 1, ix], g[iy + 1, ix + 1]
            if iy != 0:
                tris.append((a, b, d))
            if iy != h_seg - 1:
                tris.append((b, c, d))
    idx = np.array(tris, np.uint32).ravel()
    return pos.astype(np.float32), orient_outward(pos, idx)


def _superellipse(phi, e):
    c, s = np.cos(phi), np.sin(phi)
    return np.sign(c) * np.abs(c) ** (2 / e), np.sign(s) * np.abs(s) ** (2 / e)


def superellipsoid(length, width, height, stations, ring, e_xy=2.5, e_ring=3.0, seed=1, jitter=0.0):
    """Closed superellipsoid |2x/L|^e + |superellipse ring| = 1, lofted in `stations` rings of
    `ring` vertices, with end caps. Optional seeded radial jitter for surface texture."""
    rng = np.random.default_rng(seed)
    t = 0.5 - 0.5 * np.cos(np.pi * np.arange(stations + 1) / stations)  # clustered at the ends
    xs = (t - 0.5) * length
    prof = np.clip(1 - np.abs(2 * xs / length) ** e_xy, 0, 1) ** (1 / e_xy)
    prof = np.maximum(prof, 1e-3)
    phi = 2 * np.pi * np.arange(ring) / ring
    cz, cy = _superellipse(phi, e_ring)
    j = 1 + jitter * rng.standard_normal((stations + 1, ring)) if jitter else np.ones((stations + 1, ring))
    X = np.repeat(xs[:, None], ring, 1)
    Y = height / 2 * prof[:, None] * cy[None, :] * j
    Z = width / 2 * prof[:, None] * cz[None, :] * j
    pos = np.stack([X, Y, Z], -1).reshape(-1, 3)
    s, r = np.meshgrid(np.arange(stations), np.arange(ring), indexing="ij")
    a = s * ring + r
    b = s * ring + (r + 1) % ring
    c = (s + 1) * ring + r
    d = (s + 1) * ring + (r + 1) % ring
    quads = np.stack([a, c, b, b, c, d], -1).reshape(-1, 3)
    c0 = len(pos)
    c1 = c0 + 1
    pos = np.vstack([pos, pos[:ring].mean(0, keepdims=True), pos[-ring:].mean(0, keepdims=True)])
    rr = np.arange(ring)
    cap0 = np.stack([np.full(ring, c0), rr, (rr + 1) % ring], -1)
    cap1 = np.stack([np.full(ring, c1), stations * ring + (rr + 1) % ring, stations * ring + rr], -1)
    idx = np.vstack([quads, cap0, cap1]).astype(np.uint32).ravel()
    return pos, orient_outward(pos, idx)


def cylinder(radius, width, segments, centre, axis="z"):
    """Closed cylinder with `segments` sides along z, centred at `centre`."""
    phi = 2 * np.pi * np.arange(segments) / segments
    ring = np.stack([radius * np.cos(phi), radius * np.sin(phi)], -1)
    z0, z1 = -width / 2, width / 2
    pos = np.vstack([np.c_[ring, np.full(segments, z0)], np.c_[ring, np.full(segments, z1)], [[0, 0, z0], [0, 0, z1]]])
    pos = pos + np.asarray(centre, np.float64)
    k = np.arange(segments)
    k1 = (k + 1) % segments
    side = np.vstack([np.stack([k, k1, segments + k], -1), np.stack([k1, segments + k1, segments + k], -1)])
    cb, ct = 2 * segments, 2 * segments + 1
    caps = np.vstack([np.stack([np.full(segments, cb), k1, k], -1),
                      np.stack([np.full(segments, ct), segments + k, segments + k1], -1)])
    idx = np.vstack([side, caps]).astype(np.uint32).ravel()
    return pos, orient_outward(pos, idx)


def merge(parts):
    pos, idx, off = [], [], 0
    for p, i in parts:
        p = np.asarray(p, np.float64).reshape(-1, 3)
        pos.append(p)
        idx.append(np.asarray(i, np.int64).ravel() + off)
        off += len(p)
    return np.vstack(pos), np.concatenate(idx).astype(np.uint32)


def vehicle_body(target_tris=200_000, seed=1):
    """Seeded procedural vehicle: superellipsoid body (length 1, aspect 4 : 1.5 : 1.2 for
    length : width : height) raised on four 16-segment cylinder wheels of radius 0.12 * height.
    Returns (positions f32, indices u32, wheels (normalized space), min, max), normalized like
    the reference's presets (length 1 along x, lowest point on y = 0, centred in x and z)."""
    L = 1.0
    W = L * 1.5 / 4
    H = L * 1.2 / 4
    r = 0.12 * H
    ring = 256
    stations = max(8, int(round((target_tris - 4 * 64) / (2 * ring))))
    body_p, body_i = superellipsoid(L, W, H, stations, ring, seed=seed)
    body_p[:, 1] += H / 2 + r  # body floor at the wheel top
    wheels = []
    parts = [(body_p, body_i)]
    hw = 0.05 * L
    for xw in (-0.3 * L, 0.3 * L):
        for zs in (-1, 1):
            zc = zs * (W / 2 - hw * 0.6)
            cp, ci = cylinder(r, 2 * hw, 16, (xw, r, zc))
            parts.append((cp, ci))
            wheels.append({"c": [xw, r, zc], "axis": [0.0, 0.0, 1.0], "r": r, "hw": hw})
    pos, idx = merge(parts)
    p32, lo, hi, T = normalize_mesh(pos, align_longest=False)
    s = np.linalg.norm(T[:3, 0])
    wheels_n = []
    for w in wheels:
        c = apply(T, np.asarray(w["c"], np.float64))[0]
        wheels_n.append({"c": c.tolist(), "axis": w["axis"], "r": w["r"] * s, "hw": w["hw"] * s})
    return p32, idx, wheels_n, lo, hi
