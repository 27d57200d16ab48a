"""The reference's validation cases (src/analysis/validation.ts) on the CUDA path, plus
size-independent checks at the full D3Q19 benchmark size (256 x 128 x 128, FP16 storage)."""
import numpy as np
import pytest

from windtunnel_vis_b200 import validation as V
from windtunnel_vis_b200.solver import Solver, solver_factory

pytestmark = pytest.mark.gpu


def test_freestream(gpu):
    r = V.freestream(solver_factory)
    assert r["passed"], r
    assert abs(r["metrics"]["maxU_over_U"] - 1) < 1e-4 and abs(r["metrics"]["rhoRef"] - 1) < 1e-4


@pytest.mark.parametrize("prec", ["f32", "f16"])
def test_cylinder_strouhal(gpu, prec):
    # valscale 0.5 (D = 12): the oracle gives St = 0.1726, C_D = 1.501; published St 0.173
    r = V.cylinder(lambda d, p: solver_factory(d, dict(p, precision=prec)), 0.5)
    m = r["metrics"]
    assert r["passed"], m
    assert abs(m["St"] - 0.1726) < 0.003, m
    assert abs(m["cd_mean"] - 1.501) < 0.02, m


def test_sphere_drag(gpu):
    # D = 10 (valscale 0.5): within 20 % of Schiller-Naumann (validation.ts:137-184)
    r = V.sphere(solver_factory, 0.5)
    m = r["metrics"]
    assert r["passed"], m
    assert 1.15 < m["cd"] < 1.40, m


def test_full_size_fp16_against_fp32(gpu):
    # 256 x 128 x 128 sphere D = 24 (the benchmark workload): FP16 shifted storage tracks FP32
    dims = (256, 128, 128)
    flags, frontal, sdf = V.round_flags(dims, (64, 64.37, 64.21), 12, False)
    out = {}
    for prec in ("f32", "f16"):
        s = Solver(dims, dict(u=0.05, nu=0.05 * 24 / 300, cs=0.1, ground="freeslip", sides="freeslip",
                              spongeNu=0.03, spongeStart=0.85, emaAlpha=0, precision=prec))
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        st = s.step_and_sample(400)
        assert not st["unstable"]
        out[prec] = (st, s.read_velocity())
        s.destroy()
    (a, va), (b, vb) = out["f32"], out["f16"]
    fluid = flags == 0
    assert np.abs(va[fluid, :3] - vb[fluid, :3]).max() < 2e-3 * 0.05 + 1e-4
    assert abs(a["fx"] - b["fx"]) < 1e-2 * abs(a["fx"])


def test_full_size_determinism(gpu):
    dims = (256, 128, 128)
    flags, frontal, sdf = V.round_flags(dims, (64, 64.37, 64.21), 12, False)
    sums = []
    for _ in range(2):
        s = Solver(dims, dict(u=0.05, nu=0.004, cs=0.1, ground="freeslip", sides="freeslip", spongeNu=0.03,
                              spongeStart=0.85, emaAlpha=0, precision="f16", init="rest_noise", initSeed=1))
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        st = s.step_and_sample(100)
        f = s.read_populations().view(np.uint16)
        sums.append((int(f.astype(np.uint64).sum()), st["fx"]))
        s.destroy()
    assert sums[0] == sums[1]
