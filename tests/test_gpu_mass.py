"""The global mass-conservation check (an extension of the sampling pass: the FP64 sum of every
fluid cell's density, returned beside the reference's 8-slot statistics).

A closed box conserves mass exactly in exact arithmetic: a solid frame on every face of the domain
(so no cell pulls from the inlet, the outlet or a face rule), halfway bounce-back on the frame and
on a solid sphere, no inlet sponge and no moving walls. The check must see FP64 runs conserve mass
to round-off and FP32 / FP16 runs to their storage rounding, and it must equal the oracle's sum on
the same populations. (Free-slip faces that meet a solid plane are not conservative: the
reference's rules mirror a corner link onto the solid cell's stored rest state, and the check
shows that leak, about 4e-6 of the mass over 300 steps in this box.)
"""
import numpy as np
import pytest

from windtunnel_vis_b200 import validation as V
from windtunnel_vis_b200.solver import Solver

pytestmark = pytest.mark.gpu

# relative drift of the fluid mass over the run (storage rounding per step, accumulated)
DRIFT = {"f64": 1e-12, "f32": 2e-5, "f16": 3e-4}
# the GPU's sum against the oracle's on the same stored populations: per-cell densities agree to a
# few f32 ulps, summed in FP64
SAME_STATE = {"f64": 1e-13, "f32": 3e-7, "f16": 3e-7}


def closed_box(dims):
    nx, ny, nz = dims
    is3 = nz > 1
    flags, _, _ = V.round_flags(dims, (nx * 0.45, ny / 2 + 0.37, nz / 2 + 0.21 if is3 else 0), ny * 0.2, not is3)
    flags = flags.reshape(nz, ny, nx)
    flags[:, :, 0] = 1
    flags[:, :, nx - 1] = 1
    flags[:, 0, :] = 1
    flags[:, ny - 1, :] = 1
    if is3:
        flags[0] = 1
        flags[nz - 1] = 1
    return flags.ravel().astype(np.uint32)


PARAMS = dict(u=0.05, nu=0.02, cs=0.1, ground="freeslip", sides="freeslip", spongeNu=0.02, spongeStart=0.8,
              interp=False, emaAlpha=0.0, init="rest_noise", initNoise=0.02, initSeed=7)


@pytest.mark.parametrize("prec", ["f64", "f32", "f16"])
@pytest.mark.parametrize("dims", [(40, 24, 20), (96, 40, 1)])
def test_closed_box_conserves_mass(gpu, oracle, dims, prec):
    params = dict(PARAMS, precision=prec)
    flags = closed_box(dims)
    g = Solver(dims, params)
    g.upload_flags(flags)
    s0 = g.step_and_sample(1)
    fluid = int((flags == 0).sum())
    assert s0["fluidCells"] == fluid
    assert abs(s0["mass"] / fluid - 1.0) < 1e-2
    s1 = g.step_and_sample(300)
    assert not s1["unstable"] and s1["fluidCells"] == fluid
    drift = abs(s1["mass"] - s0["mass"]) / s0["mass"]
    assert drift <= DRIFT[prec], f"{prec}: mass drift {drift:.3e} over 300 steps"
    # the same stored state through the oracle's sampling pass
    o = oracle.OracleSolver(dims, params)
    o.upload_flags(flags)
    o.pending_init = False
    o.a[:] = g.read_populations()
    so = o.sample()
    assert so["fluidCells"] == fluid
    assert abs(s1["mass"] - so["mass"]) <= SAME_STATE[prec] * so["mass"], (s1["mass"], so["mass"])
    g.destroy()


def test_open_tunnel_mass_follows_oracle(gpu, oracle):
    """With an inlet and an outlet the fluid mass changes; the check tracks the oracle's run."""
    dims = (48, 20, 16)
    params = dict(PARAMS, precision="f64", interp=True, init="freestream")
    flags, _, sdf = V.round_flags(dims, (18.0, 10.37, 8.21), 4.0, False)
    g = Solver(dims, params)
    o = oracle.OracleSolver(dims, params)
    for s in (g, o):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
    for _ in range(3):
        sg, so = g.step_and_sample(40), o.step_and_sample(40)
        assert sg["fluidCells"] == so["fluidCells"]
        assert abs(sg["mass"] - so["mass"]) <= 1e-12 * so["mass"]
    g.destroy()
