"""CUDA path (through libwt.so) against the CPU oracle on the same seeded inputs.

The scalar kernel (one cell per thread: every pull rule in cell_general, the collision in
collide_full) evaluates the reference's expressions in the WGSL order, one rounding per operation
(the LBM unit is compiled without FMA contraction), as the oracle does: its populations are
bit-identical to the oracle's in every precision. Tolerances for the vectorised kernels, which
compute the same algebra rearranged (shifted populations f - w, pairwise moment sums, fused
multiply-adds where the source writes them), so single-precision results differ by a few ulp per
step:
  f64 populations ............ |Δ| <= 1e-12 after 1 and 30 steps
  f32 populations ............ |Δ| <= 1e-6 after 1 step, <= 2e-5 after 30 steps
  f16 (f - w) populations .... |Δ| <= 2e-5 after 1 step (about 2 half ulps), <= 3e-4 after 30
  force sum / max|u|² ........ relative 1e-4 (f32), 5e-3 (f16: a one-ulp f32 difference can flip
                                the rounding of a stored half, and the force sums hundreds of
                                wall links), 1e-10 (f64); counts exact
  EMA means .................. relative 1e-4 (f32, f64), 5e-3 (f16)
  reference-plane density .... absolute 1e-5 (f32, f64), 5e-5 (f16)
  fluid mass (FP64 sum) ...... relative 1e-12 (f64), 1e-6 (f32), 2e-5 (f16); fluid count exact
  velocity field ............. absolute 2e-6 (f32, f64), 1e-4 (f16)
  voxelizer flags, sdf, info . bit-exact (compiled without contraction)
  tracers .................... bit-exact state and trail
"""
import numpy as np
import pytest

from windtunnel_vis_b200 import abi, mesh as Mh
from windtunnel_vis_b200.solver import Solver, WtError

from .scenes import PARAM_SETS, scene

pytestmark = pytest.mark.gpu

TOL = {"f64": (1e-12, 1e-12), "f32": (1e-6, 2e-5), "f16": (2e-5, 3e-4)}
STAT_RTOL = {"f64": 1e-10, "f32": 1e-4, "f16": 5e-3}
MEAN_TOL = {"f64": (1e-4, 1e-7), "f32": (1e-4, 1e-7), "f16": (5e-3, 5e-5)}
VEL_ATOL = {"f64": 2e-6, "f32": 2e-6, "f16": 1e-4}  # f16: a few half ulps of ~10 populations
MASS_RTOL = {"f64": 1e-12, "f32": 1e-6, "f16": 2e-5}  # FP64 sum of the fluid densities


def _pair(oracle, dims, params):
    flags, sdf, wheels = scene(dims)
    g = Solver(dims, params)
    o = oracle.OracleSolver(dims, params)
    for s in (g, o):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        s.set_wheels(wheels)
    return g, o, flags


def _as_float(a):
    return a.astype(np.float64)


# (kernel, param, bx, by): 1 / 2 / 4 cells per thread, explicit and default block shapes
# (8, 2, 0, rows): the row pipeline (3-D tunnels with nx % 8 == 0; the others run the vectorised kernel)
LAUNCHES = {"reg1": (0, 1, 0, 0), "reg2": (0, 2, 32, 4), "reg4": (0, 4, 32, 4), "reg2d": (0, 2, 0, 0),
            "hint4": (4, 2, 0, 0), "rows2": (8, 2, 0, 2)}
CASES = [(p, k) for p in ("f32", "f16") for k in LAUNCHES] + [("f64", "reg1")]


@pytest.mark.parametrize("prec,launch", CASES)
@pytest.mark.parametrize("pset", list(PARAM_SETS))
@pytest.mark.parametrize("dims", [(32, 14, 12), (34, 14, 10), (48, 16, 1), (160, 12, 1)])
def test_stream_collide_matches_oracle(gpu, oracle, dims, pset, prec, launch):
    _check_against_oracle(oracle, dims, dict(PARAM_SETS[pset], precision=prec), LAUNCHES[launch])


def _check_against_oracle(oracle, dims, params, launch):
    prec = params["precision"]
    g, o, flags = _pair(oracle, dims, params)
    g.set_launch(*launch)
    assert g.get_launch() == launch
    t1, t30 = TOL[prec]
    # the scalar kernel (one cell per thread, collide_full) evaluates the reference's expressions in
    # the reference's order, operation by operation, like the oracle: the same bits
    exact = launch == LAUNCHES["reg1"]
    g.step(1)
    o.step(1)
    if exact:
        np.testing.assert_array_equal(g.read_populations(), o.current)
    d1 = np.abs(_as_float(g.read_populations()) - _as_float(o.current)).max()
    assert d1 <= t1, f"1 step: max |diff| {d1:.3e}"
    g.step(29)
    o.step(29)
    if exact:
        np.testing.assert_array_equal(g.read_populations(), o.current)
    d30 = np.abs(_as_float(g.read_populations()) - _as_float(o.current)).max()
    assert d30 <= t30, f"30 steps: max |diff| {d30:.3e}"
    # macro pass: stats, velocity field, EMA statistics
    sg, so = g.sample(), o.sample()
    rt = STAT_RTOL[prec]
    scale = max(np.abs(so["raw"][:3]).max(), 1e-3)
    assert np.abs(sg["raw"][:3] - so["raw"][:3]).max() <= rt * scale + 1e-9, (sg["raw"], so["raw"])
    assert abs(sg["raw"][3] - so["raw"][3]) <= rt * so["raw"][3] + 1e-12
    assert abs(sg["rhoRef"] - so["rhoRef"]) <= (5e-5 if prec == "f16" else 1e-5)
    assert sg["raw"][5:].tolist() == so["raw"][5:].tolist()
    assert sg["step"] == so["step"] == 30 and not sg["unstable"]
    # global mass-conservation check (extension): FP64 sum of the fluid cells' densities
    assert sg["fluidCells"] == so["fluidCells"] == int((flags == 0).sum())
    assert abs(sg["mass"] - so["mass"]) <= MASS_RTOL[prec] * so["mass"], (sg["mass"], so["mass"])
    vg = g.read_velocity()
    vo = o.vel.reshape(-1, 4)
    np.testing.assert_allclose(vg, vo, rtol=2e-3, atol=VEL_ATOL[prec])
    ma, mb = g.read_means()
    mr, ma_tol = MEAN_TOL[prec]
    np.testing.assert_allclose(ma, o.meanA.reshape(-1, 4), rtol=mr, atol=ma_tol)
    np.testing.assert_allclose(mb, o.meanB, rtol=max(mr, 1e-3), atol=ma_tol * 1e-2)
    g.destroy()


def test_solid_cells_and_init(gpu, oracle):
    dims = (16, 8, 8)
    params = dict(PARAM_SETS["freeslip_reg"], precision="f32")
    g, o, flags = _pair(oracle, dims, params)
    # before any step the init runs on first access, equal to the oracle's equilibrium
    o._init()
    np.testing.assert_allclose(g.read_populations(), o.current, atol=1e-7)
    g.step(3)
    f = g.read_populations().reshape(19, -1)
    solid = flags != 0
    w = oracle.lattice(3)["w"].astype(np.float32)
    np.testing.assert_array_equal(f[:, solid], np.repeat(w[:, None], solid.sum(), 1))


def test_determinism_and_checkpoint(gpu):
    dims = (32, 16, 16)
    flags, sdf, wheels = scene(dims)
    params = dict(PARAM_SETS["belt_periodic_les"], precision="f16")
    runs = []
    for _ in range(2):
        s = Solver(dims, params)
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        s.set_wheels(wheels)
        s.step(20)
        runs.append((s, s.read_populations()))
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
    # resume from a checkpoint into a fresh handle: same trajectory
    a = runs[0][0]
    b = Solver(dims, params)
    b.upload_flags(flags)
    b.upload_sdf(sdf)
    b.set_wheels(wheels)
    b.write_populations(runs[0][1])
    a.step(7)
    b.step(7)
    np.testing.assert_array_equal(a.read_populations(), b.read_populations())


def test_reset_restarts_from_init(gpu):
    dims = (24, 12, 1)
    s = Solver(dims, dict(u=0.05, nu=0.02))
    s.step(1)
    first = s.read_populations()
    s.step(10)
    s.reset()
    assert s.step_count == 0
    s.step(1)
    np.testing.assert_array_equal(s.read_populations(), first)


def test_autotune_keeps_state(gpu):
    dims = (64, 32, 24)
    flags, sdf, wheels = scene(dims)
    params = dict(PARAM_SETS["belt_periodic_les"], precision="f16")
    a, b = Solver(dims, params), Solver(dims, params)
    for s in (a, b):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        s.set_wheels(wheels)
        s.step(5)
    shape = a.autotune(3)
    # occupancy hint or the row pipeline (8, with 2..8 rows per block), cells per thread
    assert shape[0] in (0, 2, 3, 4, 8) and shape[1] in (1, 2, 4)
    if shape[0] == 8:
        assert shape[1] == 2 and shape[2] == 0 and shape[3] in (2, 4, 8)
    a.step(5)
    b.step(5)
    np.testing.assert_allclose(a.read_populations().astype(np.float32), b.read_populations().astype(np.float32),
                               atol=3e-4)


@pytest.mark.parametrize("prec", ["f32", "f16"])
def test_raw_write_and_geometry_change_follow_oracle(gpu, oracle, prec):
    # solid cells are read as stored (mirror images on the faces) until a step rewrites them; a
    # raw population write and a mid-run change of the body must give the oracle's results
    dims = (32, 14, 12)
    params = dict(PARAM_SETS["belt_periodic_les"], precision=prec)
    g, o, flags = _pair(oracle, dims, params)
    g.set_launch(3, 2, 32, 4)
    g.step(4)
    o.step(4)
    f = g.read_populations().reshape(19, -1).copy()
    rng = np.random.default_rng(5)
    solid = flags != 0
    f[:, solid] = (rng.random((19, int(solid.sum()))) * 0.01).astype(f.dtype)
    g.write_populations(f.ravel())
    o.a[:] = f.ravel()
    t1, t30 = TOL[prec]
    for k in range(3):
        g.step(1)
        o.step(1)
        d = np.abs(_as_float(g.read_populations()) - _as_float(o.current)).max()
        assert d <= t30, f"step {k + 1} after the write: max |diff| {d:.3e}"
    moved = np.roll(flags.reshape(dims[::-1]), 2, axis=2).ravel()
    for s in (g, o):
        s.upload_flags(moved)
    g.step(5)
    o.step(5)
    d = np.abs(_as_float(g.read_populations()) - _as_float(o.current)).max()
    assert d <= t30, f"after the geometry change: max |diff| {d:.3e}"
    g.destroy()


def test_errors_are_reported(gpu):
    s = Solver((16, 8, 4), dict(u=0.05, nu=0.02))
    with pytest.raises(WtError):
        s.set_launch(0, 3)
    with pytest.raises(WtError) as e:
        s.upload_flags(np.zeros(10, np.uint32))
    assert e.value.code == abi.WT_E_INVALID
    with pytest.raises(WtError):
        s.set_params(dict(precision="f16"))
    with pytest.raises(WtError):
        Solver((0, 8, 8), dict(u=0.05, nu=0.02))
    for bad in ((1, 2), (5, 2), (4, 4), (0, 2, 48, 2), (0, 2, 128, 4),  # hint, cells, block shape
                (8, 4), (8, 2, 32, 1), (8, 2, 0, 17)):  # row pipeline: cells, block, rows per block
        with pytest.raises(WtError):
            s.set_launch(*bad)


@pytest.mark.parametrize("prec", ["f16", "f32"])
@pytest.mark.parametrize("pset", ["belt_periodic_les", "noslip_bgk_halfway"])
@pytest.mark.parametrize("rows", [1, 3, 8, 16])
def test_row_pipeline_matches_vectorised_kernel(gpu, prec, pset, rows):
    """The row pipeline (rows streamed through shared memory by bulk copies) applies the vectorised
    kernel's arithmetic to the same pulled populations: 20 steps of both give the same bits (the
    LBM unit is compiled without FMA contraction, so each kernel rounds as the source is written).
    22 x 18 interior rows do not divide by 3, 8 or 16, so the last block is partial."""
    dims = (64, 24, 20)
    params = dict(PARAM_SETS[pset], precision=prec)
    flags, sdf, wheels = scene(dims)
    runs = []
    for launch in ((0, 2, 0, 0), (8, 2, 0, rows)):
        g = Solver(dims, params)
        g.upload_flags(flags)
        g.upload_sdf(sdf)
        g.set_wheels(wheels)
        g.set_launch(*launch)
        g.step(20)
        runs.append(_as_float(g.read_populations()))
        assert not g.sample()["unstable"]
        g.destroy()
    np.testing.assert_array_equal(runs[0], runs[1])


@pytest.mark.parametrize("rows", [1, 4])
def test_row_pipeline_second_x_pass(gpu, oracle, rows):
    """nx = 320 with FP16 storage: each consumer thread takes x0 = 2 tid and x0 + 256, so the
    second pass of the consumer loop (class byte reloaded, stage read at x0 + 256) runs; checked
    against the oracle and against the vectorised kernel."""
    dims = (320, 12, 10)
    params = dict(PARAM_SETS["belt_periodic_les"], precision="f16")
    flags, sdf, wheels = scene(dims)
    o = oracle.OracleSolver(dims, params)
    for s_ in (o,):
        s_.upload_flags(flags)
        s_.upload_sdf(sdf)
        s_.set_wheels(wheels)
    o.step(10)
    runs = []
    for launch in ((0, 2, 0, 0), (8, 2, 0, rows)):
        g = Solver(dims, params)
        g.upload_flags(flags)
        g.upload_sdf(sdf)
        g.set_wheels(wheels)
        g.set_launch(*launch)
        assert g.get_launch() == launch
        g.step(10)
        runs.append(_as_float(g.read_populations()))
        g.destroy()
    assert np.abs(runs[0] - runs[1]).max() <= 2e-5
    assert np.abs(runs[1] - _as_float(o.current)).max() <= TOL["f16"][1]


def test_row_pipeline_consumer_timeout_is_reported(gpu):
    """Consumer waits that give up at once (a poll limit of 0) while the producer's copies are in
    flight: the blocks store nothing, drain their copies and set bit 8 of the error word, which the
    next sample reports as WT_E_CUDA; with the default limit restored the handle steps cleanly."""
    dims = (64, 24, 20)
    params = dict(PARAM_SETS["freeslip_reg"], precision="f16")
    flags, sdf, wheels = scene(dims)
    g = Solver(dims, params)
    g.upload_flags(flags)
    g.upload_sdf(sdf)
    g.set_wheels(wheels)
    g.set_launch(8, 2, 0, 4)
    g.step(4)
    saved = g.read_populations().copy()
    ref = g.step_and_sample(4)
    g.write_populations(saved)
    g.set_wait_limit(0)
    g.step(2)
    with pytest.raises(WtError) as e:
        g.sample()
    assert e.value.code == abi.WT_E_CUDA and "error word 8" in str(e.value)
    g.set_wait_limit(-1)
    g.write_populations(saved)
    st = g.step_and_sample(4)
    assert not st["unstable"] and st["raw"].tolist() == ref["raw"].tolist()
    g.destroy()


# ---- voxelizer -------------------------------------------------------------------------------
def _sphere(dims):
    pos, idx = Mh.uv_sphere()
    p, lo, hi, _ = Mh.normalize_mesh(pos)
    M16, _, full = Mh.placement_matrix(p, lo, hi, dims, dict(mode="center", lengthFrac=1 / 3, diamFrac=0.3, xFrac=0.35))
    return p, idx, M16, []


def _vehicle(dims, tris=20000):
    p, idx, wheels, lo, hi = Mh.vehicle_body(target_tris=tris)
    M16, _, full = Mh.placement_matrix(p, lo, hi, dims, dict(mode="ground", lengthFrac=1 / 3, diamFrac=0.3,
                                                             xFrac=0.34, rideCells=0.08 * dims[1]))
    return p, idx, M16, Mh.grid_wheels(wheels, full)


@pytest.mark.parametrize("kind,dims", [("sphere", (128, 64, 64)), ("sphere", (512, 192, 1)), ("vehicle", (96, 48, 48)),
                                       ("vehicle", (160, 64, 1))])
def test_voxelizer_bit_exact(gpu, oracle, kind, dims):
    p, idx, M16, wheels = (_sphere if kind == "sphere" else _vehicle)(dims)
    s = Solver(dims, dict(u=0.05, nu=0.02))
    info = s.voxelize(p, idx, M16, wheels)
    fo, so, io = oracle.voxelize_f32(dims, p, idx, M16, wheels)
    assert info == io
    np.testing.assert_array_equal(s.read_flags(), fo)
    np.testing.assert_array_equal(s.read_sdf_encoded(), so)
    if wheels and dims[2] > 1:
        assert ((s.read_flags() >> 8) != 0).sum() > 0
    # empty mesh clears the geometry
    info0 = s.voxelize(np.zeros((0, 3), np.float32), np.zeros(0, np.uint32), M16)
    assert info0["solidCells"] == 0 and s.read_flags().sum() == 0


@pytest.mark.parametrize("prec", ["f16", "f32"])
def test_steps_after_voxelize_follow_oracle(gpu, oracle, prec):
    # the voxelizer's scratch lives in the population buffer the next step overwrites: stepping on
    # after a voxelization must give the oracle's populations from the same state and geometry
    dims = (64, 32, 24)
    params = dict(PARAM_SETS["freeslip_reg"], precision=prec, init="rest_noise", initNoise=0.01)
    s = Solver(dims, params)
    s.step(5)
    f0 = s.read_populations()
    p, idx, M16, wheels = _sphere(dims)
    s.voxelize(p, idx, M16, wheels)
    o = oracle.OracleSolver(dims, params)
    o.upload_flags(s.read_flags())
    o.sdf[:] = s.read_sdf_encoded()
    o.pending_init = False
    o.a[:] = f0
    t1, t30 = TOL[prec]
    for k in (1, 2, 5):
        s.step(k)
        o.step(k)
        d = np.abs(_as_float(s.read_populations()) - _as_float(o.current)).max()
        assert d <= t30, f"max |diff| {d:.3e}"
    s.destroy()


# ---- derived fields and export ---------------------------------------------------------------
@pytest.mark.parametrize("dims", [(40, 18, 14), (64, 24, 1)])
def test_derived_fields_and_export_bit_exact(gpu, oracle, dims):
    flags, sdf, wheels = scene(dims)
    s = Solver(dims, dict(PARAM_SETS["belt_periodic_les"], precision="f32"))
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    s.set_wheels(wheels)
    for _ in range(4):
        s.step_and_sample(10)  # EMA statistics with alpha 0.1
    s.derive_fields()
    vort, stat, mean = s.read_derived()
    vel = s.read_velocity().astype(np.float16)
    ma, mb = s.read_means()
    ov, os_, om = oracle.derive(dims, s.kparams().u_ref, vel, flags, ma, mb)
    np.testing.assert_array_equal(vort, ov.astype(np.float32))
    np.testing.assert_array_equal(stat, os_.astype(np.float32))
    np.testing.assert_array_equal(mean, om.astype(np.float32))
    fluid = flags == 0
    assert np.abs(vort[fluid, :3]).max() > 0 and (stat[~fluid, 1] == 1).all() and (stat[fluid, 1] == 0).all()
    for stride in (1, 2, 3, 7):
        e = s.export_fields(stride)
        r = oracle.export(dims, stride, vel, om, ov)
        assert e["dims"] == r["dims"] and e["stride"] == stride
        for k in ("vel", "mean", "vort"):
            np.testing.assert_array_equal(e[k], r[k], err_msg=f"{k} stride {stride}")
    s.destroy()


def test_backend_export_stride(gpu):
    from windtunnel_vis_b200.solver import Backend

    b = Backend()
    b.create_solver((64, 32, 16), dict(u=0.05, nu=0.02))
    b.frame(4)
    n = 64 * 32 * 16
    for max_points, stride in ((n, 1), (n // 8, 2), (n // 8 - 1, 3), (1000, 4)):
        e = b.export_fields(max_points)
        assert e["stride"] == stride
        assert e["vel"].shape[0] == np.prod(e["dims"]) and e["dims"] == tuple(-(-d // stride) for d in (64, 32, 16))
    b.destroy()


@pytest.mark.parametrize("dims", [(48, 24, 16), (64, 32, 1)])
def test_streamlines_and_probes_bit_exact(gpu, oracle, dims):
    flags, sdf, wheels = scene(dims)
    s = Solver(dims, dict(PARAM_SETS["freeslip_reg"], init="rest_noise", initNoise=0.02))
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    for _ in range(3):
        s.step_and_sample(20)
    vel = s.read_velocity().astype(np.float16)
    u_lat = s.kparams().uin
    for use_mean in (0, 1):
        sp = abi.StreamlineParams(seeds=3 * 14, points=120, use_mean=use_mean, per_line=14)
        sp.rake_a[:] = [3.0, 2.0, 2.0, 0.0]
        sp.rake_b[:] = [3.0, dims[1] - 2.0, max(dims[2] - 2.0, 0.5), 0.0]
        sp.rake_d[:] = [0.0, 0.0, 2.5, 0.0]
        sp.h = 0.7
        pts = s.streamlines(sp)
        mean = s.read_derived()[2].astype(np.float16) if use_mean else vel
        ref = oracle.streamlines(dims, sp, u_lat, vel, mean, flags)
        np.testing.assert_array_equal(pts, ref, err_msg=f"use_mean {use_mean}")
        alive = pts[:, 3] >= 0
        assert alive.sum() > 0 and (~alive).sum() > 0  # lines advance, and some end
    pos = [(5.5, 7.25, 3.1), (20.0, 12.0, 8.0), (30.7, 3.3, 1.0)]
    pr = s.probes(pos)
    _, _, mean = s.read_derived()
    p4 = np.zeros((3, 4), np.float32)
    p4[:, :3] = pos
    ref = oracle.probes(dims, p4, vel, mean.astype(np.float16))
    got = np.array([p["inst"] + p["mean"] for p in pr], np.float32)
    np.testing.assert_array_equal(got, ref)
    s.destroy()


# ---- tracers ---------------------------------------------------------------------------------
@pytest.mark.parametrize("dims,emitter", [((48, 24, 16), 0), ((48, 24, 16), 1), ((64, 32, 1), 0), ((64, 32, 1), 1)])
def test_tracers_bit_exact(gpu, oracle, dims, emitter):
    flags, sdf, wheels = scene(dims)
    s = Solver(dims, dict(PARAM_SETS["freeslip_reg"], init="rest_noise", initNoise=0.02))
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    s.step_and_sample(40)
    vel = s.read_velocity().astype(np.float16)
    count, trail = 3000, 5
    tp = abi.TracerParams(count=count, trail=trail, head=0, emitter=emitter, steps=6.0, seed=11, max_age=12.0,
                          nozzles=7)
    tp.lines = 3
    tp.rake_a[:] = [2.0, 3.0, 1.0, 0.0]
    tp.rake_b[:] = [2.0, dims[1] - 3.0, max(dims[2] - 1.0, 0.5), 0.0]
    tp.rake_d[:] = [0.0, 0.0, 1.5, 0.0]
    st = np.zeros((count, 4), np.float32)
    hi = np.zeros((count * trail, 4), np.float32)
    for frame in range(6):
        tp.fill = 1 if frame == 0 else 0
        tp.advance = 0 if frame == 0 else 1
        tp.head = frame % trail
        tp.seed = 11 + frame
        s.advect_tracers(tp)
        oracle.tracers(dims, tp, vel, flags, st, hi)
        gs, gh = s.read_tracers(count, trail)
        np.testing.assert_array_equal(gs, st, err_msg=f"frame {frame}")
        np.testing.assert_array_equal(gh, hi, err_msg=f"frame {frame}")


# ---- batches of tunnels -----------------------------------------------------------------------
def test_batch_matches_members_stepped_alone(gpu):
    from windtunnel_vis_b200.solver import Batch

    cases = [((32, 14, 12), dict(PARAM_SETS["belt_periodic_les"], precision="f16")),
             ((48, 20, 16), dict(PARAM_SETS["freeslip_reg"], precision="f32")),
             ((64, 16, 1), dict(PARAM_SETS["noslip_bgk_halfway"], precision="f16")),
             ((36, 12, 10), dict(PARAM_SETS["freeslip_reg"], precision="f64"))]

    def make(dims, params):
        flags, sdf, wheels = scene(dims)
        s = Solver(dims, params)
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        s.set_wheels(wheels)
        return s

    batch_members = [make(d, p) for d, p in cases]
    alone = [make(d, p) for d, p in cases]
    b = Batch(batch_members)
    for steps in (7, 10, 1, 6):
        b.step(steps)
        for s in alone:
            s.step(steps)
    for s, t in zip(batch_members, alone):
        np.testing.assert_array_equal(s.read_populations(), t.read_populations())
        assert s.step_count == t.step_count == 24
    got = b.sample()
    for st, t in zip(got, alone):
        assert st["raw"].tolist() == t.sample()["raw"].tolist()
    # a member's parameters change mid-run: the batch recaptures and stays with its twin
    batch_members[1].set_params(dict(u=0.07))
    alone[1].set_params(dict(u=0.07))
    b.step(8)
    for s in alone:
        s.step(8)
    for s, t in zip(batch_members, alone):
        np.testing.assert_array_equal(s.read_populations(), t.read_populations())
    b.destroy()
    for s in batch_members + alone:
        s.destroy()


def test_reuploading_unchanged_geometry_keeps_the_classification(gpu):
    """Uploads land in a staging buffer and replace the geometry only when it differs: re-uploading
    the same flags and wall distances adds only the compare launches (the comparison and the
    hand-over of its result word; the sdf encode before the sdf comparison), and the run stays
    bit-identical to one without the re-upload."""
    dims = (48, 20, 16)
    params = dict(PARAM_SETS["freeslip_reg"], precision="f16")
    flags, sdf, wheels = scene(dims)
    a, b = Solver(dims, params), Solver(dims, params)
    for s in (a, b):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        s.set_wheels(wheels)
        s.step(12)
    la, lb = a.launches, b.launches
    a.upload_flags(flags)
    a.upload_sdf(sdf)
    a.step(12)
    b.step(12)
    assert a.launches - la == b.launches - lb + 5  # diff + take (flags), encode + diff + take (sdf)
    np.testing.assert_array_equal(a.read_populations(), b.read_populations())
    a.destroy()
    b.destroy()


def test_sdf_only_upload_refreshes_the_wall_links(gpu, oracle):
    """New wall distances alone (same flags) change the Bouzidi fractions of the link records: a run
    that switches distances mid-way matches the oracle doing the same."""
    dims = (32, 14, 12)
    params = dict(PARAM_SETS["freeslip_reg"], precision="f32")
    flags, sdf, wheels = scene(dims)
    sdf2 = np.where(sdf >= 0, np.clip(sdf * 0.6 + 0.2, 0.0, 2.4), sdf).astype(np.float32)
    g = Solver(dims, params)
    o = oracle.OracleSolver(dims, params)
    for s in (g, o):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        s.set_wheels(wheels)
        s.step(5)
        s.upload_sdf(sdf2)
        s.step(5)
    d = np.abs(g.read_populations().astype(np.float64) - o.current.astype(np.float64))
    assert d.max() <= 2e-5, d.max()
    g.destroy()


@pytest.mark.parametrize("prec", ["f32", "f16"])
def test_zero_weight_means_follow_the_oracle_with_non_finite_cells(gpu, oracle, prec):
    """With emaAlpha = 0 the sampling pass leaves the means of finite cells untouched and writes
    them only where the sample is not finite (0 x NaN = NaN), as the reference's mix() does: means
    after a sample of populations holding NaN and Inf cells match the oracle's."""
    dims = (32, 14, 12)
    params = dict(PARAM_SETS["freeslip_reg"], precision=prec, emaAlpha=0.0)
    g, o, flags = _pair(oracle, dims, params)
    g.step(4)
    o.step(4)
    pops = g.read_populations().copy()
    n = dims[0] * dims[1] * dims[2]
    fluid = np.flatnonzero(flags == 0)
    bad = fluid[[7, 300, 999]]
    pops[1 * n + bad[0]] = np.nan
    pops[2 * n + bad[1]] = np.inf
    pops[5 * n + bad[2]] = -np.inf
    g.write_populations(pops)
    o.a[:] = pops
    g.sample()
    o.sample()
    ma, mb = g.read_means()
    ma, mb = ma.reshape(-1, 4), np.asarray(mb).ravel()
    oa, ob = o.meanA.reshape(-1, 4), o.meanB
    assert np.array_equal(np.isnan(ma), np.isnan(oa)) and np.array_equal(np.isnan(mb), np.isnan(ob))
    assert np.isnan(ma[bad]).any(axis=1).all()
    ok = ~np.isnan(oa)
    assert np.array_equal(ma[ok], oa[ok])
    g.destroy()


@pytest.mark.parametrize("prec", ["f16", "f32"])
def test_fused_batch_matches_members_stepped_alone(gpu, prec):
    """Members that share storage and collision step their bulk rows in one launch of the batch
    kernel (face rows and wall cells on their own auxiliary streams): each advances exactly as it
    does alone."""
    from windtunnel_vis_b200.solver import Batch

    cases = [((32, 14, 12), dict(PARAM_SETS["belt_periodic_les"], precision=prec)),
             ((48, 20, 16), dict(PARAM_SETS["freeslip_reg"], precision=prec)),
             ((130, 18, 10), dict(PARAM_SETS["freeslip_reg"], precision=prec, u=0.04))]

    def make(dims, params):
        flags, sdf, wheels = scene(dims)
        s = Solver(dims, params)
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        s.set_wheels(wheels)
        return s

    members = [make(d, p) for d, p in cases]
    alone = [make(d, p) for d, p in cases]
    b = Batch(members, fused=True)
    l0, la0 = sum(s.launches for s in members), sum(t.launches for t in alone)
    for steps in (7, 10, 1, 6):
        b.step(steps)
        for s in alone:
            s.step(steps)
    for s, t in zip(members, alone):
        np.testing.assert_array_equal(s.read_populations(), t.read_populations())
    # the fused graph: one batch-kernel launch per step instead of one bulk launch per member
    assert sum(s.launches for s in members) - l0 < sum(t.launches for t in alone) - la0
    got = b.sample()
    for st, t in zip(got, alone):
        assert st["raw"].tolist() == t.sample()["raw"].tolist()
    b.destroy()
    for s in members + alone:
        s.destroy()


def test_half4_velocity_readback_is_the_storage_format(gpu):
    """wt_read_velocity_half4 returns the stored binary16 field; wt_read_velocity widens it."""
    dims = (32, 14, 12)
    g = Solver(dims, dict(PARAM_SETS["freeslip_reg"], precision="f16"))
    flags, sdf, wheels = scene(dims)
    g.upload_flags(flags)
    g.upload_sdf(sdf)
    g.step_and_sample(6)
    h = g.read_velocity_half()
    f = g.read_velocity()
    assert h.dtype == np.float16 and h.shape == f.shape
    np.testing.assert_array_equal(h.astype(np.float32), f)
    g.destroy()
