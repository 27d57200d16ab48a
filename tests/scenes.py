"""Small seeded scenes that switch on every boundary path of the solver at once: an interpolated
(Bouzidi) sphere / circle, a rotating wheel touching the floor, a non-wheel solid on the floor
(belt contact patches), inlet and outlet sponges, periodic or free-slip sides."""
import numpy as np

from windtunnel_vis_b200 import validation as V


def scene(dims):
    nx, ny, nz = dims
    is3 = nz > 1
    zc = nz / 2 + 0.21 if is3 else 0
    flags, _, sdf = V.round_flags(dims, (nx * 0.36, ny / 2 + 0.37, zc), min(ny, max(nz, ny)) * 0.2, not is3)
    flags = flags.reshape(nz, ny, nx)
    sdf = sdf.reshape(nz, ny, nx)
    z, y, x = np.meshgrid(np.arange(nz) + 0.5, np.arange(ny) + 0.5, np.arange(nx) + 0.5, indexing="ij")
    wc = (nx * 0.72, 2.0, nz / 2 if is3 else 0.5)
    wr, whw = 1.8, 2.0
    rad = np.sqrt((x - wc[0]) ** 2 + (y - wc[1]) ** 2)
    inside = (rad < wr) & ((np.abs(z - wc[2]) < whw) if is3 else True)
    flags[inside] = 1 | (1 << 8)
    dw = np.abs(rad - wr)
    near = (dw < 2.5) & ((np.abs(z - wc[2]) < whw + 1) if is3 else True)
    sdf = np.where(near & ((sdf < 0) | (dw < sdf)), dw, sdf).astype(np.float32)
    # a plain solid standing on the floor: holds the belt still around it
    x0 = int(nx * 0.15)
    if is3:
        flags[nz // 3:nz // 3 + 2, 0, x0:x0 + 2] = 1
    else:
        flags[0, 0, x0:x0 + 2] = 1
    wheels = [{"c": list(wc), "axis": [0.0, 0.0, 1.0], "r": wr, "hw": whw}]
    return flags.ravel().astype(np.uint32), sdf.ravel(), wheels


PARAM_SETS = {
    "belt_periodic_les": dict(u=0.05, nu=0.02, cs=0.15, ground="moving", sides="periodic", spongeNu=0.05,
                              spongeStart=0.6, spongeIn=0.1, tauWall=0.53, emaAlpha=0.1, init="rest_noise",
                              initNoise=0.01, initSeed=3),
    "noslip_bgk_halfway": dict(u=0.04, nu=0.03, cs=0.0, ground="noslip", sides="freeslip", spongeNu=0.03,
                               spongeStart=0.85, collision="bgk", interp=False, emaAlpha=0.0),
    "freeslip_reg": dict(u=0.06, nu=0.01, cs=0.1, ground="freeslip", sides="freeslip", spongeNu=0.02,
                         spongeStart=0.8, emaAlpha=0.02),
}
