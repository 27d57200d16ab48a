"""The sampling pass fused into the last step of a stepAndSample chunk (the step's kernels write the
velocity texels, EMA statistics and sums from the values they store; a short pass adds the wall
force and the solid cells) gives the same bits as the separate sampling pass (k_macro) after the
same steps: the 8 reference statistics but the force, the mass sum and fluid count, the velocity
field, the means and the populations exactly; the force sums to FP64 rounding (another summation
order over the same per-cell values). Every boundary path of the parity scenes is switched on."""
import numpy as np
import pytest

from windtunnel_vis_b200.solver import Solver

from .scenes import PARAM_SETS, scene

pytestmark = pytest.mark.gpu

CASES = [((32, 14, 12), (0, 2, 0, 0)), ((34, 14, 10), (4, 2, 0, 0)), ((32, 14, 12), (0, 4, 32, 4)),
         ((48, 16, 1), (0, 2, 0, 0)), ((160, 12, 1), (0, 4, 32, 4))]


def _pair(dims, params, launch):
    flags, sdf, wheels = scene(dims)
    out = []
    for _ in range(2):
        s = Solver(dims, params)
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        s.set_wheels(wheels)
        s.set_launch(*launch)
        out.append(s)
    return out


@pytest.mark.parametrize("prec", ["f16", "f32"])
@pytest.mark.parametrize("pset", list(PARAM_SETS))
@pytest.mark.parametrize("dims,launch", CASES)
def test_fused_sampling_matches_separate_pass(gpu, dims, launch, pset, prec):
    a, b = _pair(dims, dict(PARAM_SETS[pset], precision=prec), launch)
    for chunk in (7, 12, 1):
        sa = a.step_and_sample(chunk)
        b.step(chunk)
        sb = b.sample()
        assert sa["raw"][3:].tolist() == sb["raw"][3:].tolist(), (sa["raw"], sb["raw"])
        np.testing.assert_allclose(sa["raw"][:3], sb["raw"][:3], rtol=1e-12, atol=1e-15)
        assert sa["mass"] == sb["mass"] and sa["fluidCells"] == sb["fluidCells"]
        assert sa["step"] == sb["step"] and sa["unstable"] == sb["unstable"]
        np.testing.assert_array_equal(a.read_velocity_half(), b.read_velocity_half())
        for x, y in zip(a.read_means(), b.read_means()):
            np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(a.read_populations(), b.read_populations())
    assert a.fused_samples == 3 and b.fused_samples == 0
    a.destroy()
    b.destroy()


def test_unfused_configurations_fall_back(gpu):
    # FP64 storage (the scalar kernel) and the row pipeline run the separate pass
    dims = (64, 24, 20)
    flags, sdf, wheels = scene(dims)
    for params, launch in ((dict(PARAM_SETS["freeslip_reg"], precision="f64"), None),
                           (dict(PARAM_SETS["freeslip_reg"], precision="f16"), (8, 2, 0, 4))):
        s = Solver(dims, params)
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        if launch:
            s.set_launch(*launch)
        st = s.step_and_sample(4)
        assert not st["unstable"] and s.fused_samples == 0
        s.destroy()
