"""The reference's validation cases, driven through a solver factory.

round_flags .... src/analysis/validation.ts:35-53 (analytic circle / sphere flags + exact sdf)
freestream ..... src/analysis/validation.ts:61-88
cylinder ....... src/analysis/validation.ts:89-136
sphere ......... src/analysis/validation.ts:137-184
cylinder_channel the D2Q9 cylinder in a 512 x 128 channel of the benchmark (FP32 against FP64
                 populations)
sphere_les ..... the D3Q19 LES sphere tunnel of the benchmark (FP16 storage against FP64 populations)
vehicle ........ the D3Q19 vehicle tunnel of the benchmark (GPU voxelizer, moving belt, wheels)
batch_sweep .... 32 vehicle tunnels of uneven sizes (yaw x speed sweep) stepped as one batch
learned_closure  training data from filtered fine runs, GPU training, coarse runs with the network
                 against the fine run and plain Smagorinsky (windtunnel_vis_b200.closure.study)

A factory is any callable make(dims, params) returning an object with the LbmSolver surface
(upload_flags, upload_sdf, step_and_sample, destroy) — windtunnel_vis_b200.solver.SolverFactory
for the CUDA path. Sizes scale with `valscale` like the reference's ?valscale= query.
"""
import math
import time

import numpy as np

from .analysis import coefficients, crossing_frequency, cylinder_st_ref, sphere_cd_ref


def js_round(x):
    """Math.round: halves round towards +infinity."""
    return int(math.floor(x + 0.5))


def round_flags(dims, c, r, cylinder):
    """Analytic obstacle flags for a circle (2-D) or sphere (3-D): flags u32, frontal cell count,
    sdf f32 (distance |‖p − c‖ − r| where < 2.5, else −1), all in f64 like the reference."""
    nx, ny, nz = dims
    z, y, x = np.meshgrid(np.arange(nz, dtype=np.float64), np.arange(ny, dtype=np.float64),
                          np.arange(nx, dtype=np.float64), indexing="ij")
    dx = x + 0.5 - c[0]
    dy = y + 0.5 - c[1]
    dz = np.zeros_like(dx) if cylinder else z + 0.5 - c[2]
    r2 = dx * dx + dy * dy + dz * dz
    dist = np.abs(np.sqrt(r2) - r)
    sdf = np.where(dist < 2.5, dist, -1.0).astype(np.float32).ravel()
    inside = r2 < r * r
    flags = inside.astype(np.uint32).ravel()
    frontal = int(inside.any(axis=2).sum())
    return flags, frontal, sdf


def freestream(make, valscale=1.0):
    t0 = time.perf_counter()
    d = (256, 96, 1)
    U = 0.08
    s = make(d, dict(u=U, nu=0.01, cs=0.1, ground="freeslip", sides="freeslip", spongeNu=0.05, spongeStart=0.85,
                     emaAlpha=0.02))
    s.upload_flags(np.zeros(d[0] * d[1], np.uint32))
    st = s.step_and_sample(1)
    for _ in range(20):
        st = s.step_and_sample(50)
    s.destroy()
    err = abs(st["maxU"] - U) / U
    drho = abs(st["rhoRef"] - 1)
    return {"id": "freestream", "passed": err < 0.01 and drho < 0.01 and not st["unstable"],
            "seconds": time.perf_counter() - t0,
            "metrics": {"maxU_over_U": st["maxU"] / U, "rhoRef": st["rhoRef"]}}


def cylinder(make, valscale=1.0, interp=True):
    """interp=False: plain halfway bounce-back instead of Bouzidi walls (SolverParams.interp)."""
    t0 = time.perf_counter()
    D = js_round(24 * valscale)
    d = (js_round(25 * D), 10 * D, 1)
    U = 0.06
    Re = 100
    nu = U * D / Re
    s = make(d, dict(u=U, nu=nu, cs=0, ground="freeslip", sides="freeslip", spongeNu=0.03, spongeStart=0.85,
                     emaAlpha=0.0, interp=interp))
    flags, _, sdf = round_flags(d, (6 * D, d[1] / 2 + 0.37, 0), D / 2, True)
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    period = D / (0.17 * U)
    total = js_round(period * 16)
    measure_from = js_round(period * 6)
    chunk = max(5, js_round(period / 40))
    tt, cl, cd = [], [], []
    step = 0
    while step < total:
        st = s.step_and_sample(chunk)
        if st["unstable"]:
            break
        c = coefficients(st["fx"], st["fy"], 0, U, D)
        if step >= measure_from:
            tt.append(st["step"])
            cl.append(c["cl"])
            cd.append(c["cd"])
        step += chunk
    s.destroy()
    fr = crossing_frequency(tt, cl)
    St = fr["f"] * D / U
    cd_mean = sum(cd) / max(len(cd), 1)
    passed = (0.16 <= St <= 0.2) and fr["cycles"] >= 4
    return {"id": "cylinder", "passed": bool(passed), "seconds": time.perf_counter() - t0,
            "series": {"t": tt, "v": cl},
            "metrics": {"St": St, "St_ref": cylinder_st_ref(Re), "cd_mean": cd_mean, "cl_amplitude": fr["amplitude"],
                        "cycles": fr["cycles"], "grid": d, "tau": 3 * nu + 0.5}}


def sphere(make, valscale=1.0, interp=True):
    """interp=False: plain halfway bounce-back instead of Bouzidi walls (SolverParams.interp)."""
    t0 = time.perf_counter()
    D = js_round(20 * valscale)
    d = (js_round(9.6 * D), js_round(4.8 * D), js_round(4.8 * D))
    U = 0.05
    Re = 100
    nu = U * D / Re
    s = make(d, dict(u=U, nu=nu, cs=0, ground="freeslip", sides="freeslip", spongeNu=0.03, spongeStart=0.85,
                     emaAlpha=0, interp=interp))
    flags, frontal, sdf = round_flags(d, (2.8 * D, d[1] / 2 + 0.37, d[2] / 2 + 0.21), D / 2, False)
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    flow_through = d[0] / U
    total = js_round(flow_through * 2.2)
    measure_from = js_round(flow_through * 1.4)
    chunk = 50
    tt, cds = [], []
    step = 0
    while step < total:
        st = s.step_and_sample(chunk)
        if st["unstable"]:
            break
        c = coefficients(st["fx"], st["fy"], st["fz"], U, frontal)
        tt.append(st["step"])
        cds.append(c["cd"])
        step += chunk
    s.destroy()
    sel = [v for t, v in zip(tt, cds) if t >= measure_from]
    cd = sum(sel) / max(len(sel), 1)
    ref = sphere_cd_ref(Re)
    err = (cd - ref) / ref
    return {"id": "sphere", "passed": abs(err) < 0.2, "seconds": time.perf_counter() - t0,
            "series": {"t": tt, "v": cds},
            "metrics": {"cd": cd, "cd_ref": ref, "deviation": err, "grid": d, "frontal": frontal,
                        "blockage": frontal / (d[1] * d[2])}}


CHANNEL_DIMS = (512, 128, 1)


def channel_params(precision="f32", u=0.05, re=100.0, diameter=20, sponge_nu=0.0, seed=1):
    """The D2Q9 cylinder-in-a-channel parameters: plain BGK (cs = 0), nu = u D / Re (0.01 at the
    defaults, tau = 0.53), free-slip floor and roof, zero-gradient outlet (with an outlet sponge
    only when sponge_nu > 0; the reference's own cylinder case uses 0.03 from 0.85 nx), rest state
    with seeded uniform +-1e-4 velocity noise."""
    return dict(u=u, nu=u * diameter / re, cs=0.0, ground="freeslip", sides="freeslip", spongeNu=sponge_nu,
                spongeStart=0.85, collision="bgk", emaAlpha=0.0, precision=precision, init="rest_noise",
                initNoise=1e-4, initSeed=seed)


def channel_geometry(dims=CHANNEL_DIMS, center=(96.0, 65.0), diameter=20):
    """Circle of diameter D centred at `center` in cell-centre coordinates (cell k spans [k, k+1],
    its centre at k + 1/2, as the reference's roundFlags), one cell above the channel axis; wall
    distances from the exact circle."""
    return round_flags(dims, (center[0], center[1], 0.0), diameter / 2, True)


def cylinder_channel(make, precision="f32", steps=40000, dims=CHANNEL_DIMS, center=(96.0, 65.0), diameter=20,
                     u=0.05, re=100.0, chunk=50, sponge_nu=0.0, seed=1, measure_from=None, init="rest_noise"):
    """The D2Q9 cylinder in a channel: 512 x 128, D = 20 at (96, 65) (one cell off the axis, which
    triggers shedding), uniform inlet u = 0.05, Re = 100, channel_params, 40,000 steps sampled every
    50. Reports the Strouhal number from upward mean crossings of C_L (the reference's estimator,
    src/analysis/strouhal.ts:5-30), mean C_D and the C_L amplitude over the steps from
    `measure_from` (default: the second half), with C = F / (1/2 rho U^2 D) as the reference's 2-D
    coefficients (src/analysis/aero.ts:4-7)."""
    t0 = time.perf_counter()
    flags, _, sdf = channel_geometry(dims, center, diameter)
    s = make(dims, dict(channel_params(precision, u, re, diameter, sponge_nu, seed), init=init))
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    tt, cl, cd, mass, rho_ref = [], [], [], [], []
    step = 0
    unstable = False
    while step < steps:
        st = s.step_and_sample(chunk)
        step += chunk
        if st["unstable"]:
            unstable = True
            break
        c = coefficients(st["fx"], st["fy"], 0, u, diameter)
        tt.append(st["step"])
        cl.append(c["cl"])
        cd.append(c["cd"])
        mass.append(st.get("mass", math.nan))
        rho_ref.append(st["rhoRef"])
    # the inflow the body actually sees: mean x velocity over the reference plane x = refX (4)
    u_in = math.nan
    if hasattr(s, "read_velocity"):
        v = np.asarray(s.read_velocity(), np.float64).reshape(dims[1], dims[0], 4)
        u_in = float(v[:, min(4, dims[0] - 1), 0].mean())
    s.destroy()
    start = steps // 2 if measure_from is None else measure_from
    sel = [k for k, t in enumerate(tt) if t >= start]
    fr = crossing_frequency([tt[k] for k in sel], [cl[k] for k in sel])
    St = fr["f"] * diameter / u
    cd_mean = sum(cd[k] for k in sel) / max(len(sel), 1)
    return {"id": "cylinder_channel", "precision": precision,
            "passed": bool(not unstable and fr["cycles"] >= 4),
            "seconds": time.perf_counter() - t0,
            "series": {"t": tt, "cl": cl, "cd": cd, "mass": mass, "rhoRef": rho_ref},
            "metrics": {"St": St, "St_ref": cylinder_st_ref(re), "cd_mean": cd_mean, "cl_amplitude": fr["amplitude"],
                        "cycles": fr["cycles"], "steps": step, "measured_from": start, "grid": list(dims),
                        "tau": 3 * u * diameter / re + 0.5, "sponge_nu": sponge_nu, "unstable": unstable,
                        "rho_ref_end": rho_ref[-1] if rho_ref else math.nan, "u_inflow_end": u_in,
                        "St_inflow": fr["f"] * diameter / u_in if u_in == u_in and u_in > 0 else math.nan,
                        "mass_end": mass[-1] if mass else math.nan}}


def sphere_les(make, precision="f16", steps=20000, dims=(256, 128, 128), diameter=24, u=0.05, re=300.0, cs=0.1,
               seed=1, chunk=50, measure_from=None):
    """Sphere in a D3Q19 LES tunnel: diameter 24 at (64, 64.37, 64.21) (off-axis by fractions of a
    cell like the reference's sphere case), inlet u = 0.05, Re = 300, Smagorinsky Cs = 0.1,
    rest state with seeded 1e-4 velocity noise. Returns the C_D / C_L / C_S series and the mean
    C_D with its batch-means standard error over the steps from `measure_from` (default: the
    second half). Run it with precision "f16" (shifted FP16 storage) and "f64" (FP64 populations
    on the GPU, the plain method's reference run) to state the storage error."""
    from .analysis import window_stats

    t0 = time.perf_counter()
    nu = u * diameter / re
    p = dict(u=u, nu=nu, cs=cs, ground="freeslip", sides="freeslip", spongeNu=0.03, spongeStart=0.85, emaAlpha=0,
             precision=precision, init="rest_noise", initNoise=1e-4, initSeed=seed)
    flags, frontal, sdf = round_flags(dims, (64.0, 64.37, 64.21), diameter / 2, False)
    s = make(dims, p)
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    tt, cd, cl, cz = [], [], [], []
    step = 0
    unstable = False
    while step < steps:
        st = s.step_and_sample(chunk)
        step += chunk
        if st["unstable"]:
            unstable = True
            break
        c = coefficients(st["fx"], st["fy"], st["fz"], u, frontal)
        tt.append(st["step"])
        cd.append(c["cd"])
        cl.append(c["cl"])
        cz.append(c["cs"])
    s.destroy()
    start = steps // 2 if measure_from is None else measure_from
    sel = [k for k, t in enumerate(tt) if t >= start]
    ws = window_stats([tt[k] for k in sel], [cd[k] for k in sel], float(steps)) if len(sel) >= 16 else None
    amp = lambda v: (max(v[k] for k in sel) - min(v[k] for k in sel)) / 2 if sel else math.nan
    return {"id": "sphere_les", "precision": precision, "passed": not unstable and ws is not None,
            "seconds": time.perf_counter() - t0, "series": {"t": tt, "cd": cd, "cl": cl, "cs": cz},
            "metrics": {"cd_mean": ws["mean"] if ws else math.nan, "cd_se": ws["se"] if ws else math.nan,
                        "cl_amplitude": amp(cl), "cs_amplitude": amp(cz), "steps": step, "measured_from": start,
                        "frontal": frontal, "grid": list(dims), "nu": nu, "unstable": unstable}}


def vehicle_setup(dims=(512, 256, 256), target_tris=200_000, seed=1):
    """The vehicle-like body of the benchmark: seeded superellipsoid body (length nx / 3, aspect
    4 : 1.5 : 1.2) on four 16-segment wheels of radius 0.12 * height, about 200k triangles,
    placed on the floor with a ride height of 0.08 * body height (the reference app's placement,
    mode 'ground', at x = 0.34 nx). Returns (positions, indices, column-major matrix, grid-space
    wheels, body height in cells)."""
    from . import mesh as Mh

    p, idx, wheels, lo, hi = Mh.vehicle_body(target_tris=target_tris, seed=seed)
    scale = dims[0] / 3.0  # lengthFrac 1/3 of a unit-length mesh
    height = float(hi[1] - lo[1]) * scale
    M16, _, full = Mh.placement_matrix(p, lo, hi, dims, dict(mode="ground", lengthFrac=1 / 3, diamFrac=0.3,
                                                             xFrac=0.34, rideCells=0.08 * height))
    return p, idx, M16, Mh.grid_wheels(wheels, full), height


def vehicle(make, precision="f16", steps=30000, dims=(512, 256, 256), u=0.06, re_l=1e6, cs=0.14, chunk=100,
            measure_from=None):
    """Vehicle tunnel: the body of vehicle_setup voxelized on the GPU (solver.voxelize), moving
    belt at the inlet speed, rotating wheels, Re_L = 1e6 on the body length with Smagorinsky LES
    (Cs 0.14, the reference app's default), rest initial state with seeded noise. Reports mean
    C_D / C_L (frontal area from the voxelizer) with batch-means errors over the second half."""
    from .analysis import window_stats

    t0 = time.perf_counter()
    p, idx, M16, wheels, height = vehicle_setup(dims)
    length = dims[0] / 3.0
    nu = u * length / re_l
    params = dict(u=u, nu=nu, cs=cs, ground="moving", sides="freeslip", spongeNu=0.03, spongeStart=0.85,
                  emaAlpha=0, precision=precision, init="rest_noise", initNoise=1e-4, initSeed=1)
    s = make(dims, params)
    info = s.voxelize(p, idx, M16, wheels)
    t_vox = time.perf_counter() - t0
    tt, cd, cl = [], [], []
    step = 0
    unstable = False
    while step < steps:
        st = s.step_and_sample(chunk)
        step += chunk
        if st["unstable"]:
            unstable = True
            break
        c = coefficients(st["fx"], st["fy"], st["fz"], u, info["frontal"])
        tt.append(st["step"])
        cd.append(c["cd"])
        cl.append(c["cl"])
    s.destroy()
    start = steps // 2 if measure_from is None else measure_from
    sel = [k for k, t in enumerate(tt) if t >= start]
    wd = window_stats([tt[k] for k in sel], [cd[k] for k in sel], float(steps)) if len(sel) >= 16 else None
    wl = window_stats([tt[k] for k in sel], [cl[k] for k in sel], float(steps)) if len(sel) >= 16 else None
    return {"id": "vehicle", "precision": precision, "passed": not unstable and wd is not None,
            "seconds": time.perf_counter() - t0, "series": {"t": tt, "cd": cd, "cl": cl},
            "metrics": {"cd_mean": wd["mean"] if wd else math.nan, "cd_se": wd["se"] if wd else math.nan,
                        "cl_mean": wl["mean"] if wl else math.nan, "cl_se": wl["se"] if wl else math.nan,
                        "voxel": info, "triangles": int(np.asarray(idx).size // 3), "body_height_cells": height,
                        "tau0": 3 * nu + 0.5, "steps": step, "unstable": unstable, "setup_seconds": t_vox}}


def sweep_cases(count=32):
    """The batched sweep: `count` tunnels of uneven sizes from 128 x 64 x 64 to 384 x 192 x 192
    (nx a multiple of 4), yaw -10 to +10 degrees in 8 steps x inlet u in {0.03, 0.04, 0.05, 0.06}
    around the vehicle body. Returns [(dims, yaw, u)]."""
    yaws = [-10.0 + 20.0 * k / 7 for k in range(8)]
    us = [0.03, 0.04, 0.05, 0.06]
    out = []
    for k in range(count):
        sc = 1.0 + 2.0 * k / max(count - 1, 1)
        d = (int(round(128 * sc / 4)) * 4, int(round(64 * sc)), int(round(64 * sc)))
        out.append((d, yaws[k % 8], us[(k // 8) % 4]))
    return out


def batch_sweep(steps=10000, count=32, chunk=250, compare_alone=False, cs=0.14, re_l=2e4, target_tris=200_000,
                closure=None, fused=False, autotune=True, persistent=False, queue=False):
    """Runs the sweep of sweep_cases as one batch (windtunnel_vis_b200.solver.Batch): every tunnel
    voxelizes the vehicle body at its yaw (moving belt, rotating wheels, Smagorinsky LES, FP16),
    then all advance `steps` lattice updates together. Reports the aggregate MLUPS (device time
    of the batch steps) and each case's mean C_D / C_L over the second half; with compare_alone,
    the same cases stepped one tunnel at a time (each with its own CUDA graphs) for the speed-up
    and the per-case C_D, which must agree exactly (the batch replays the same kernels). `closure`
    (a network, see windtunnel_vis_b200.closure) replaces Smagorinsky in every tunnel; with
    `autotune` the project's launch tuner picks each tunnel's block shape and cells per thread;
    `persistent` runs each batch step call as one launch of the persistent kernel over all tunnels;
    `queue` runs each step of all tunnels as one launch of that kernel's work queue, under the batch
    graphs."""
    import torch

    from . import mesh as Mh
    from .analysis import window_stats
    from .solver import Batch, Solver

    p, idx, wheels, lo, hi = Mh.vehicle_body(target_tris=target_tris)
    cases = sweep_cases(count)

    def build():
        solvers, frontal = [], []
        for dims, yaw, u in cases:
            length = dims[0] / 3.0
            s = Solver(dims, dict(u=u, nu=u * length / re_l, cs=cs, ground="moving", sides="freeslip", spongeNu=0.03,
                                  spongeStart=0.85, emaAlpha=0, precision="f16", init="rest_noise", initNoise=1e-4,
                                  initSeed=1))
            body_h = float(hi[1] - lo[1]) * length
            M16, _, full = Mh.placement_matrix(p, lo, hi, dims, dict(mode="ground", lengthFrac=1 / 3, diamFrac=0.3,
                                                                     xFrac=0.34, yawDeg=yaw, rideCells=0.08 * body_h))
            info = s.voxelize(p, idx, M16, Mh.grid_wheels(wheels, full))
            if closure is not None:
                s.set_closure(closure)
            elif autotune:
                s.autotune(6)
            frontal.append(max(info["frontal"], 1))
            solvers.append(s)
        return solvers, frontal

    def run(step_fn, sample_fn, frontal):
        series = [[] for _ in cases]
        ms = 0.0
        done = 0
        torch.cuda.synchronize()
        while done < steps:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            step_fn(chunk)
            b.record()
            torch.cuda.synchronize()
            ms += a.elapsed_time(b)
            done += chunk
            for k, st in enumerate(sample_fn()):
                series[k].append((st["step"], coefficients(st["fx"], st["fy"], st["fz"], cases[k][2], frontal[k])))
        res = []
        for k, ser in enumerate(series):
            sel = [(t, c) for t, c in ser if t > steps // 2]
            w = window_stats([t for t, _ in sel], [c["cd"] for _, c in sel], float(steps)) if len(sel) >= 16 else None
            res.append({"dims": list(cases[k][0]), "yaw": cases[k][1], "u": cases[k][2],
                        "cd": float(np.mean([c["cd"] for _, c in sel])) if sel else math.nan,
                        "cd_se": w["se"] if w else math.nan,
                        "cl": float(np.mean([c["cl"] for _, c in sel])) if sel else math.nan})
        return ms, res

    cells = sum(d[0] * d[1] * d[2] for d, _, _ in cases)
    solvers, frontal = build()
    batch = Batch(solvers, fused=fused, persistent=persistent, queue=queue)

    def step_batch(n):
        batch.step(n)
        torch.cuda.synchronize()  # the batch stream is not torch's: wait before the end event

    ms, res = run(step_batch, batch.sample, frontal)
    out = {"id": "batch_sweep", "tunnels": count, "cells": cells, "steps": steps, "closure": closure is not None,
           "fused": fused, "persistent": persistent, "queue": queue, "autotune": autotune and closure is None,
           "batch_ms": ms,
           "batch_mlups": cells * steps / (ms * 1e-3) / 1e6, "cases": res}
    batch.destroy()
    for s in solvers:
        s.destroy()
    if compare_alone:
        solvers, frontal = build()

        def step_alone(n):
            for s in solvers:  # one tunnel at a time
                s.step(n)
                torch.cuda.synchronize()

        ms2, res2 = run(step_alone, lambda: [s.sample() for s in solvers], frontal)
        out["alone_ms"] = ms2
        out["alone_mlups"] = cells * steps / (ms2 * 1e-3) / 1e6
        out["cd_identical"] = all(a["cd"] == b["cd"] for a, b in zip(res, res2))
        for s in solvers:
            s.destroy()
    return out


CASES = {"freestream": freestream, "cylinder": cylinder, "sphere": sphere}


def main(argv=None):
    """python -m windtunnel_vis_b200.validation sphere_les --precision f16 --steps 20000
    python -m windtunnel_vis_b200.validation cylinder_channel --precision f32 --steps 40000
    python -m windtunnel_vis_b200.validation vehicle --precision f16 --steps 30000
    python -m windtunnel_vis_b200.validation cylinder|sphere|freestream [--valscale 0.5]
    Prints one JSON line (metrics, series omitted) per case on the CUDA path."""
    import argparse
    import json

    from .solver import solver_factory

    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["sphere_les", "vehicle", "batch_sweep", "learned_closure", "cylinder_channel",
                                     *CASES])
    ap.add_argument("--precision", default="f16")
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--sponge", type=float, default=0.0, help="cylinder_channel: outlet sponge viscosity")
    ap.add_argument("--valscale", type=float, default=1.0)
    ap.add_argument("--fine", default="512,256,256", help="learned_closure: fine grid nx,ny,nz")
    ap.add_argument("--train-bodies", type=int, default=8)
    ap.add_argument("--eval-bodies", type=int, default=2)
    ap.add_argument("--warm", type=int, default=6000)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--keep", type=float, default=0.4)
    ap.add_argument("--re", type=float, default=1000.0)
    ap.add_argument("--radius", type=int, default=1, help="learned_closure: projection box half-width")
    ap.add_argument("--height", type=float, default=0.125, help="learned_closure: body height / tunnel height")
    ap.add_argument("--save", default=None, help="learned_closure: write the trained network (.npz)")
    ap.add_argument("--fused", action="store_true", help="batch_sweep: bulk rows of all tunnels in one kernel")
    ap.add_argument("--persistent", action="store_true", help="batch_sweep: all tunnels' steps in one persistent launch")
    ap.add_argument("--queue", action="store_true", help="batch_sweep: each step of all tunnels in one work-queue launch")
    ap.add_argument("--outside-regime", action="store_true",
                    help="batch_sweep: apply --closure outside its stored Reynolds-number regime (throughput only)")
    ap.add_argument("--closure", default=None,
                    help="batch_sweep: a network (.npz) or 'pretrained' in place of Smagorinsky in every tunnel")
    a = ap.parse_args(argv)
    if a.case == "learned_closure":
        from . import closure as CL

        fine = tuple(int(v) for v in a.fine.split(","))
        r = CL.study(solver_factory, fine_dims=fine, train_bodies=a.train_bodies, eval_bodies=a.eval_bodies,
                     warm=a.warm, train_steps=a.train_steps, keep=a.keep, re=a.re, eval_steps=a.steps, radius=a.radius,
                     height=a.height, log=lambda m: print(m, flush=True))
        if a.save:
            # gated to a factor of two around the Reynolds number it was trained and checked at
            CL.save({k: np.asarray(v, np.float32) for k, v in r["model"].items()}, a.save,
                    regime={"re": (a.re / 2.0, a.re * 2.0)})
        r.pop("model", None)
        print(json.dumps(r, default=float), flush=True)
        return
    if a.case == "sphere_les":
        r = sphere_les(solver_factory, a.precision, a.steps)
    elif a.case == "cylinder_channel":
        r = cylinder_channel(solver_factory, a.precision, a.steps, sponge_nu=a.sponge)
    elif a.case == "vehicle":
        r = vehicle(solver_factory, a.precision, a.steps)
    elif a.case == "batch_sweep":
        model = None
        if a.closure:
            from . import closure as CL

            # the vehicle tunnels run at Re_L = 2e4 on the body length, 6720 on its height (0.336 of
            # the length): outside the shipped network's regime, allowed only for throughput runs
            model = CL.load_pretrained(2e4 * 0.336, allow_outside=a.outside_regime,
                                       path=CL.PRETRAINED if a.closure == "pretrained" else a.closure)
        r = batch_sweep(a.steps, compare_alone=True, closure=model, fused=a.fused, persistent=a.persistent,
                        queue=a.queue)
    else:
        r = CASES[a.case](solver_factory, a.valscale)
    r.pop("series", None)
    print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
