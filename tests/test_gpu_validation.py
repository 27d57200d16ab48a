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
    # valscale 0.5 (D = 12), Bouzidi walls: the oracle gives St = 0.1726, C_D = 1.501
    r = V.cylinder(lambda d, p: solver_factory(d, dict(p, precision=prec)), 0.5)
    m = r["metrics"]
    assert r["passed"], m
    assert abs(m["St"] - 0.1726) < 0.003, m
    assert abs(m["cd_mean"] - 1.501) < 0.02, m


def test_cylinder_published_run(gpu):
    # the reference's published cylinder result (README.md:175): St = 0.173 from its D = 18 run
    # (valscale 0.75), C_D about 1.5. The published table predates the reference's Bouzidi walls
    # (README.md:262-264: they moved its D = 10 sphere from +23 % to +15 %), so the pin is the
    # halfway bounce-back run; the Bouzidi run lands within the same margin.
    for interp in (False, True):
        m = V.cylinder(solver_factory, 0.75, interp=interp)["metrics"]
        assert abs(m["St"] - 0.173) <= 0.003, (interp, m)
        assert abs(m["cd_mean"] - 1.5) <= 0.05, (interp, m)


@pytest.mark.parametrize("valscale,interp,cd_pub", [(0.5, False, 1.342), (0.7, False, 1.250),
                                                    (0.5, True, 1.09173 * 1.15)])
def test_sphere_published_runs(gpu, valscale, interp, cd_pub):
    # the reference's published sphere drag (README.md:176): 1.342 at D = 10 (+23 %) and 1.250 at
    # D = 14 (+14.5 %) with halfway bounce-back, and +15 % at D = 10 with Bouzidi walls
    # (README.md:262-264), against Schiller-Naumann 1.0917 (validation.ts:137-184)
    r = V.sphere(solver_factory, valscale, interp=interp)
    m = r["metrics"]
    assert abs(m["cd"] / cd_pub - 1) <= 0.01, m


def test_channel_cylinder_fp32_against_fp64_populations(gpu):
    # the D2Q9 cylinder in a 512 x 128 channel (D = 20 at (96, 65), u = 0.05, Re = 100, BGK, rest
    # state with seeded noise, 40,000 steps sampled every 50): FP32 populations against the FP64
    # run of the same method on the GPU, St within 1 % and mean C_D within 0.5 %
    r32 = V.cylinder_channel(solver_factory, "f32")
    r64 = V.cylinder_channel(solver_factory, "f64")
    m32, m64 = r32["metrics"], r64["metrics"]
    assert r32["passed"] and r64["passed"], (m32, m64)
    assert abs(m32["St"] / m64["St"] - 1) <= 1e-2, (m32, m64)
    assert abs(m32["cd_mean"] / m64["cd_mean"] - 1) <= 5e-3, (m32, m64)
    # from rest, the reference's equilibrium inlet (incoming populations at rho = 1, u = U) and the
    # zero-gradient outlet settle where 3 rho* u* = 1 + 3 U - rho*: rho* about 1.039, u* about
    # 0.74 U; on that inflow the shedding frequency is the unconfined cylinder's (St about 0.167)
    assert abs(m64["rho_ref_end"] - 1.0388) < 2e-3 and abs(m64["u_inflow_end"] / 0.05 - 0.735) < 0.02, m64
    assert abs(m64["St_inflow"] - 0.167) < 0.005, m64


def test_channel_cylinder_matches_oracle_full_size(gpu, oracle):
    # the same channel at full size, 300 steps from rest on both paths, then the sampling pass
    dims = V.CHANNEL_DIMS
    params = V.channel_params("f32")
    flags, _, sdf = V.channel_geometry()
    g = Solver(dims, params)
    o = oracle.OracleSolver(dims, params)
    for s in (g, o):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
    g.step(300)
    o.step(300)
    d = np.abs(g.read_populations().astype(np.float64) - o.current.astype(np.float64)).max()
    assert d <= 1e-5, d
    sg, so = g.sample(), o.sample()
    # the force is a sum over the cylinder's ~400 wall links of about 2 f each; after 300 steps the
    # two runs' populations differ by ~1e-7 typically (1e-5 at most), so the sums may differ by a
    # few 1e-6 in every component. The drag is 1.5e-2; the lift cancels to ~5e-5 this early, so the
    # bound is absolute: 5e-6, 3e-4 of the drag
    assert np.abs(sg["raw"][:3] - so["raw"][:3]).max() <= 5e-6, (sg["raw"][:3], so["raw"][:3])
    assert abs(sg["raw"][0] / so["raw"][0] - 1) <= 2e-4
    assert sg["raw"][5:].tolist() == so["raw"][5:].tolist()
    # the two runs' f32 roundings differ (the GPU's rearranged algebra against the WGSL order) and the
    # collision's rounding moves mass a little every step: the mass sums agree to the drift of
    # 300 rounded steps (the sum itself is checked on identical populations in test_gpu_mass)
    assert sg["fluidCells"] == so["fluidCells"] and abs(sg["mass"] / so["mass"] - 1) <= 2e-5
    g.destroy()


@pytest.mark.parametrize("case", ["channel_f32", "sphere_tunnel_f16"])
def test_scalar_kernel_bit_identical_to_oracle_full_size(gpu, oracle, case):
    # the scalar kernel evaluates the reference's expressions in the reference's order: at full size
    # its populations equal the oracle's bit for bit (the D2Q9 channel, FP32, 300 steps from rest;
    # the benchmark's sphere tunnel, FP16 shifted storage, Smagorinsky, 10 steps)
    import bench

    if case == "channel_f32":
        dims, params, steps = V.CHANNEL_DIMS, V.channel_params("f32"), 300
        flags, _, sdf = V.channel_geometry()
    else:
        dims, params, steps = bench.DIMS, bench.PARAMS, 10
        flags, _, sdf = bench.geometry()
    g = Solver(dims, params)
    o = oracle.OracleSolver(dims, params)
    for s in (g, o):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
    g.set_launch(0, 1, 0, 0)
    g.step(steps)
    o.step(steps)
    np.testing.assert_array_equal(g.read_populations(), o.current)
    g.destroy()


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


def test_sphere_les_f16_tracks_f64_populations(gpu):
    # the benchmark's sphere tunnel from rest: FP16 shifted storage shadows the FP64-population run
    # through the first 1000 steps; afterwards half-precision rounding, amplified by the start-up
    # pressure waves in this nearly inviscid LES (tau0 = 0.512), makes the instantaneous drag drift
    # (up to 10 % by step 2500), so only the means over steps 1500-3000 are compared (3 %)
    r16 = V.sphere_les(solver_factory, "f16", steps=3000, measure_from=1500)
    r64 = V.sphere_les(solver_factory, "f64", steps=3000, measure_from=1500)
    assert r16["passed"] and r64["passed"]
    c16, c64 = np.array(r16["series"]["cd"]), np.array(r64["series"]["cd"])
    assert np.abs(c16[:20] - c64[:20]).max() <= 1e-2 * np.abs(c64[:20]).max()
    assert abs(r16["metrics"]["cd_mean"] / r64["metrics"]["cd_mean"] - 1) < 3e-2


def test_benchmark_tunnel_matches_oracle(gpu, oracle):
    # the bench workload itself (256 x 128 x 128, FP16, sphere D = 24, LES) against the oracle's
    # restatement of the reference's FP16 path: 60 steps (populations within the FP16 step
    # tolerance: a one-ulp f32 difference flips the rounding of a stored half now and then), then the macro
    # pass on identical populations
    import bench

    flags, _, sdf = bench.geometry()
    g = Solver(bench.DIMS, bench.PARAMS)
    o = oracle.OracleSolver(bench.DIMS, bench.PARAMS)
    for s in (g, o):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
    g.step(60)
    o.step(60)
    d = np.abs(g.read_populations().astype(np.float64) - o.current.astype(np.float64))
    assert d.max() <= 3e-4, d.max()
    # the macro pass on identical populations: force sums (FP64 over thousands of wall links),
    # counts and the reference-plane density
    g.write_populations(o.current)
    sg, so = g.sample(), o.sample()
    # the force is a sum of ~1e4 wall-link terms of size ~0.05 that cancel to ~5e-4 this early; one
    # f32 ulp per term (3.7e-9, the GPU's summation order against the oracle's) bounds the
    # difference at ~1e-6, far below the terms themselves
    assert np.abs(sg["raw"][:3] - so["raw"][:3]).max() <= 1e-6
    assert sg["raw"][5:].tolist() == so["raw"][5:].tolist()
    assert abs(sg["rhoRef"] - so["rhoRef"]) <= 1e-6
    g.destroy()


def test_vehicle_voxelization_full_size(gpu, oracle):
    # the benchmark's vehicle body (about 200k triangles) into 512 x 256 x 256: flags, wall
    # distances and the info block bit-exact against the f32 restatement of the reference's GPU
    # voxelizer, and cell for cell against the f64 restatement of its CPU voxelizer
    dims = (512, 256, 256)
    p, idx, M16, wheels, _ = V.vehicle_setup(dims)
    s = Solver(dims, dict(u=0.06, nu=1e-5, cs=0.14, ground="moving", precision="f16"))
    info = s.voxelize(p, idx, M16, wheels)
    fo, so, io = oracle.voxelize_f32(dims, p, idx, M16, wheels)
    assert info == io
    flags = s.read_flags()
    np.testing.assert_array_equal(flags, fo)
    np.testing.assert_array_equal(s.read_sdf_encoded(), so)
    assert ((flags >> 8) != 0).sum() > 0  # wheel cells tagged
    f64, sdf64, info64 = oracle.voxelize_f64(dims, p, idx, M16)
    assert info64["solidCells"] == info["solidCells"] and info64["frontal"] == info["frontal"]
    np.testing.assert_array_equal((flags & 1) != 0, f64 != 0)
    k = so != 0
    both = k & (sdf64 >= 0)
    assert np.abs((~so[both]).view(np.float32) - sdf64[both]).max() < 1e-4
    # a distance is kept below 2.5 cells; f32 and f64 may land on either side of that cut
    odd = np.flatnonzero(k != (sdf64 >= 0))
    assert odd.size <= 8
    d_odd = np.where(k[odd], (~so[odd]).view(np.float32), sdf64[odd])
    assert np.all(np.abs(d_odd - 2.5) < 1e-4), d_odd
    s.destroy()


def test_vehicle_tunnel_runs(gpu):
    # the vehicle tunnel (moving belt, rotating wheels, Re_L = 1e6 LES, FP16) stays stable and
    # gives a positive drag over its first 1000 steps
    r = V.vehicle(solver_factory, "f16", steps=1000, chunk=25, measure_from=500)
    m = r["metrics"]
    assert r["passed"], m
    assert not m["unstable"] and np.isfinite(m["cd_mean"]) and m["cd_mean"] > 0
