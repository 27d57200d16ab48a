"""Benchmark: D3Q19 lattice updates per second on the sphere tunnel.

Workload (one bench step = one reference sample chunk, stepAndSample(50)): 50 fused pull-stream +
collide steps of a 256 x 128 x 128 D3Q19 tunnel (FP16 shifted population storage, f32
arithmetic, Smagorinsky Cs = 0.1, regularized BGK) around a sphere of diameter 24 at (64, 64, 64)
with Bouzidi walls, inlet u = 0.05, Re = 300 (nu = 0.004), rest initial state with seeded 1e-4
velocity noise; the last step also runs the sampling pass (velocity field, EMA statistics, FP64
mass and reference-plane sums) on the values it stores, followed by the momentum-exchange force
of the wall cells and the 80-byte statistics readback.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` = lattice updates (all ranks) / device time of the timed steps (CUDA events, max over
ranks). `e2e` = the same metric through the public API with host buffers: every step uploads the
body's flags and wall distances from pinned host memory, runs stepAndSample(50) and reads the
velocity field back in its storage format (rgba16float, 8 B per cell) into pinned memory, with the
queued calls (the upload of the next step and the readback of the last one overlap the current
chunk on the handle's copy streams; the clock stops after the last readback). `roofline` =
algorithmic bytes of one stream-collide launch
(19 x (2 + 2) B per cell) over its mean duration, timed with events on the solver's stream.
Multi-GPU: independent tunnel replicas, one per rank (no data-path collective).
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DIMS = (256, 128, 128)
CHUNK = 50
TAIL = 10  # steps of the captured chunk tail in wt_step_and_sample (WT_SAMPLE_TAIL)
U = 0.05
D = 24
PARAMS = dict(u=U, nu=U * D / 300, cs=0.1, ground="freeslip", sides="freeslip", spongeNu=0.03, spongeStart=0.85,
              emaAlpha=0.0, precision="f16", init="rest_noise", initNoise=1e-4, initSeed=1)
BYTES_PER_UPDATE = 19 * 2 * 2  # D3Q19, FP16: each population read once and written once
METRIC = "D3Q19 MLUPS"
WORKLOAD = "D3Q19 sphere tunnel 256x128x128, FP16 shifted storage, Smagorinsky Cs=0.1, Bouzidi, Re=300"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_traffic(shape, closure=False):
    """DRAM bytes (read + write) per step of this launch shape (cells per thread, block) from the
    committed ncu summary (steady state: three consecutive launches of each step kernel), or None
    when that shape was not captured. The occupancy hint changes the register allocation, not the
    loads and stores, so it is not part of the key."""
    name = "stream_collide_d3q19_f16_sphere256_learned_closure.md" if closure else "stream_collide_d3q19_f16_sphere256.md"
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    cells, bx, by = (int(v) for v in shape[1:])
    if bx == 0 and by == 0 and cells > 1:
        # the default block of the vectorised kernel: one row of up to 128 threads
        runs = DIMS[0] // cells
        bx, by = (128 if runs >= 128 else ((runs + 31) // 32) * 32), 1
    key = "lc" if closure else f"{cells},{bx},{by}"
    for m in re.finditer(r"^traffic_bytes_per_step\[([0-9a-z,]+)\]:\s*(\d+)", open(p).read(), flags=re.M):
        if m.group(1) == key:
            return int(m.group(2))
    return None


def bench_closure():
    """A seeded network for timing the learned-closure step, its input normalisation set to the
    bench tunnel's feature ranges (timing does not depend on the weights' values)."""
    from windtunnel_vis_b200 import closure as CL

    scale = 1.0 / np.array([2e-4, 2e-4, 2e-4, 1e-4, 1e-4, 1e-4, 2e-3, 1.0, 2e-3, 0.02])
    return CL.init_model(seed=1, shift=[0, 0, 0, 0, 0, 0, 1e-3, 2.5, 1.0, 0.05], scale=scale, nu_scale=2e-4)


def geometry():
    from windtunnel_vis_b200.validation import round_flags

    return round_flags(DIMS, (64, 64.37, 64.21), D / 2, False)


class Clocks:
    """SM clock and clock-event reasons of this rank's GPU, sampled every 10 ms by a host thread
    through NVML for as long as the `with` block runs (the timed region): the same counters as
    `nvidia-smi --query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.*`, without a process
    start-up that can outlast a short timed region. Falls back to an nvidia-smi sampler."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.thread = None
        self.rows = []
        self.mx = None
        self.path = os.path.join(tempfile.gettempdir(), f"wt_bench_clocks_rank{index}_{os.getpid()}.csv")

    def _nvml_start(self):
        import threading

        import pynvml
        import torch

        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.index).uuid)
        h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        self.mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        bits = (pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap)
        self.stop = threading.Event()

        def run():
            while not self.stop.is_set():
                sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                r = int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.rows.append((sm, tuple(bool(r & b) for b in bits)))
                self.stop.wait(0.01)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def __enter__(self):
        try:
            self._nvml_start()
        except Exception:
            self.thread = None
            try:
                self.fh = open(self.path, "w")
                self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                              "--format=csv", "-lms", "50"], stdout=self.fh, stderr=subprocess.DEVNULL)
            except (OSError, FileNotFoundError):
                self.proc = None
        return self

    def __exit__(self, *a):
        if self.thread:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)
            self.fh.close()

    def summary(self):
        if self.thread:
            rows, mx, source = self.rows, self.mx, "nvml, 10 ms"
        elif self.proc:
            with open(self.path) as fh:
                raw = [r.split(", ") for r in fh.read().strip().split("\n")[1:] if r.strip()]
            os.remove(self.path)
            rows = [(float(r[1].split()[0]), tuple(r[5 + k].strip() == "Active" for k in range(4))) for r in raw]
            mx = float(raw[0][2].split()[0]) if raw else None
            source = "nvidia-smi, 50 ms"
        else:
            return None
        if not rows:
            return None
        sm = [v for v, _ in rows]
        reasons = sorted({self.NAMES[k] for _, r in rows for k in range(4) if r[k]})
        loaded = [v for v in sm if v > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows),
                "source": source}


def cpu_port_mlups(seconds=12.0, threads=0, steps_cap=None):
    """The oracle (CPU restatement of the reference's shader) on the same workload, all host
    threads, bounded to about `seconds` of work. Returns (MLUPS, threads, steps run)."""
    from oracle import oracle as O

    th = O.threads(threads)
    flags, _, sdf = geometry()
    s = O.OracleSolver(DIMS, PARAMS)
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    s.step(1)  # init + warm-up
    n = DIMS[0] * DIMS[1] * DIMS[2]
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds and (steps_cap is None or done < steps_cap):
        s.step(1)
        done += 1
    dt = time.perf_counter() - t0
    return n * done / dt / 1e6, th, done


def max_over_ranks(dist, v):
    """The slowest rank's time (ms or s): an all-reduce MAX over the process group (a CUDA tensor
    for NCCL, a CPU one for gloo); v itself with one process."""
    if dist is None:
        return v
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_mlups(world, cells, updates, ms):
    """Whole-job lattice updates per second over `world` independent tunnels of `cells` cells,
    each advanced `updates` steps in `ms` milliseconds (the slowest rank's time), in MLUPS."""
    return world * cells * updates / (ms / 1e3) / 1e6


def components(s, peak, no_cpu):
    """Timings of the other kernels on the path, rank 0 at N = 1 (each with its CPU restatement
    timed beside it on the host cores):
      sample ..... the macro pass (force, EMA statistics, velocity field) on the bench tunnel;
                   91 B per cell: 19 x 2 B populations, flags, class byte, 16 + 4 B EMA read and
                   written, 8 B velocity
      derive ..... the derived-field pass on the bench tunnel; 56 B per cell: velocity 8 B,
                   flags 4 B, EMA 16 + 4 B read, three binary16 x 4 fields written
      tracers .... 150,000 particles, trail 20, 50 lattice steps per frame, 18 nozzles (the
                   reference app's 3-D settings), advected through the bench tunnel's velocity
                   field; 48 B per particle (state read and written, one trail point)
      voxelize ... the vehicle body (about 200k triangles) into 512 x 256 x 256 through the public
                   API (host mesh in, flags / wall distances / info on the device); 24 B per cell
                   (3 i32 crossing counters, vote word, flags, wall distance)
      closure_step the bench tunnel's stream-collide step with the learned closure in place of
                   Smagorinsky; 76 B per update as the headline, plus 3072 tensor-core flops per
                   cell (x' W1 with K padded to 16, then h1 W2)
    """
    import torch

    from oracle import oracle as O
    from windtunnel_vis_b200 import abi
    from windtunnel_vis_b200.solver import Solver
    from windtunnel_vis_b200.validation import vehicle_setup

    n = DIMS[0] * DIMS[1] * DIMS[2]
    st = torch.cuda.ExternalStream(s.stream)
    out = {}

    def timed(fn, reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        a.record(st)
        for _ in range(reps):
            fn()
        b.record(st)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps, (time.perf_counter() - t0) * 1e3 / reps

    # macro pass
    ms, wall = timed(s.sample, 10)
    alg = n * 91
    out["sample"] = {"ms": round(ms, 4), "e2e_ms": round(wall, 4), "bytes_alg": alg,
                     "achieved_gbs": round(alg / ms / 1e6, 1), "frac": round(alg / ms / 1e6 / peak, 4)}

    # derived fields (vorticity, Q, turbulence intensity, binary16 mean)
    s.derive_fields()
    ms, wall = timed(s.derive_fields, 10)
    alg = n * 56
    out["derive"] = {"ms": round(ms, 4), "bytes_alg": alg, "achieved_gbs": round(alg / ms / 1e6, 1),
                     "frac": round(alg / ms / 1e6 / peak, 4)}

    # streamlines (the reference app's 3-D setting: 700 points per line, step 0.7, a 3 x 24 rake)
    from windtunnel_vis_b200 import abi as A

    sp = A.StreamlineParams(seeds=3 * 24, points=700, use_mean=0, per_line=24)
    sp.rake_a[:] = [4.0, 40.0, 40.0, 0.0]
    sp.rake_b[:] = [4.0, 88.0, 88.0, 0.0]
    sp.rake_d[:] = [0.0, 0.0, 6.0, 0.0]
    sp.h = 0.7
    ms, wall = timed(lambda: s.streamlines(sp), 5)
    out["streamlines"] = {"ms": round(ms, 4), "e2e_ms": round(wall, 4), "lines": sp.seeds, "points": sp.points}
    probes = [(64.0 + 20 * k, 64.0, 64.0) for k in range(8)]
    ms, wall = timed(lambda: s.probes(probes), 10)
    out["probes"] = {"ms": round(ms, 4), "e2e_ms": round(wall, 4), "count": len(probes)}
    if not no_cpu:
        vel16 = s.read_velocity().astype(np.float16)
        _, _, mean = s.read_derived()
        flags_all = np.asarray(geometry()[0], np.uint32)
        t0 = time.perf_counter()
        O.streamlines(DIMS, sp, s.kparams().uin, vel16, mean.astype(np.float16), flags_all)
        out["streamlines"]["cpu_ref_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
        ma, mb = s.read_means()
        t0 = time.perf_counter()
        O.derive(DIMS, s.kparams().u_ref, vel16, flags_all, ma, mb)
        out["derive"]["cpu_ref_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
        out["derive"]["cpu_threads"] = O.threads(0)
        # the macro pass restated on the host (one sample of the same tunnel)
        t0 = time.perf_counter()
        oo = O.OracleSolver(DIMS, PARAMS)
        oo.upload_flags(flags_all)
        oo.upload_sdf(geometry()[2])
        oo.pending_init = False
        oo.a[:] = s.read_populations()
        t1 = time.perf_counter()
        oo.sample()
        out["sample"]["cpu_ref_ms"] = round((time.perf_counter() - t1) * 1e3, 2)
        out["sample"]["cpu_threads"] = O.threads(0)

    # tracers
    count, trail, steps = 150000, 20, float(CHUNK)
    tp = abi.TracerParams(count=count, trail=trail, head=0, emitter=0, steps=steps, seed=7,
                          max_age=min(max(1.2 * DIMS[0] / max(U * steps, 1e-3), 60.0), 6000.0), nozzles=18)
    tp.fill, tp.advance = 1, 0
    s.advect_tracers(tp)
    tp.fill, tp.advance = 0, 1
    frame = [0]

    def advect():
        frame[0] += 1
        tp.head = frame[0] % trail
        tp.seed = 7 + frame[0]
        s.advect_tracers(tp)

    ms, wall = timed(advect, 20)
    out["tracers"] = {"ms": round(ms, 4), "e2e_ms": round(wall, 4), "particles": count, "trail": trail,
                      "mparticles_per_s": round(count / ms / 1e3, 1), "bytes_alg": count * 48,
                      "achieved_gbs": round(count * 48 / ms / 1e6, 1)}
    if not no_cpu:
        vel = s.read_velocity().astype(np.float16)
        flags = np.asarray(geometry()[0], np.uint32)
        state, hist = s.read_tracers(count, trail)
        state, hist = state.copy(), hist.copy()
        tp.head = (frame[0] + 1) % trail
        t0 = time.perf_counter()
        O.tracers(DIMS, tp, vel, flags, state, hist)
        out["tracers"]["cpu_ref_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
        out["tracers"]["cpu_kind"] = "port"
        out["tracers"]["cpu_threads"] = O.threads(0)

    # learned closure: the stream-collide step of the bench tunnel with the network in place of
    # Smagorinsky (bulk kernel with the two 32-wide layers on tcgen05), its own handle
    from windtunnel_vis_b200 import closure as CL

    flags_c, _, sdf_c = geometry()
    c = Solver(DIMS, PARAMS)
    c.upload_flags(flags_c)
    c.upload_sdf(sdf_c)
    c.set_closure(bench_closure())
    c.step(20)
    cst = torch.cuda.ExternalStream(c.stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # ten-step calls replay the long step graph, as a stepAndSample chunk does
    reps = 8
    torch.cuda.synchronize()
    a.record(cst)
    for _ in range(reps):
        c.step(10)
    b.record(cst)
    torch.cuda.synchronize()
    cms = a.elapsed_time(b) / (10 * reps)
    out["closure_step"] = {"ms_per_update": round(cms, 4), "mlups": round(n / cms / 1e3, 1),
                           "bytes_alg": n * 76, "achieved_gbs": round(n * 76 / cms / 1e6, 1),
                           "frac": round(n * 76 / cms / 1e6 / peak, 4),
                           "tensor_flop_per_cell": 2 * (16 * 32 + 32 * 32),
                           "tensor_tflops": round(2 * (16 * 32 + 32 * 32) * n / cms / 1e9, 2)}
    c.destroy()
    if not no_cpu:
        oc = O.OracleSolver(DIMS, PARAMS)
        oc.upload_flags(flags_c)
        oc.upload_sdf(sdf_c)
        oc.set_closure(CL.to_struct(CL.init_model(seed=1, nu_scale=2e-4)))
        oc._init()
        t0 = time.perf_counter()
        oc.step(1)
        out["closure_step"]["cpu_ref_ms"] = round((time.perf_counter() - t0) * 1e3, 1)
        out["closure_step"]["cpu_threads"] = O.threads(0)

    out["d2q9_cylinder"] = d2q9_cylinder(peak, no_cpu)
    # the same channel through the persistent multi-step kernel (one cooperative launch per call)
    from windtunnel_vis_b200 import abi as A

    out["d2q9_cylinder_persistent"] = d2q9_cylinder(peak, True, launch=(A.WT_LAUNCH_PERSISTENT, 2, 0, 0))
    # and through the work queue, one launch per step under the step graphs
    out["d2q9_cylinder_queue"] = d2q9_cylinder(peak, True, launch=(A.WT_LAUNCH_QUEUE, 2, 0, 0))

    # voxelizer (vehicle config, its own 512 x 256 x 256 handle)
    vd = (512, 256, 256)
    p, idx, M16, wheels, _ = vehicle_setup(vd)
    v = Solver(vd, dict(u=0.06, nu=1e-5, cs=0.14, ground="moving", precision="f16"))
    v.voxelize(p, idx, M16, wheels)
    vst = torch.cuda.ExternalStream(v.stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a.record(vst)
    reps = 5
    for _ in range(reps):
        info = v.voxelize(p, idx, M16, wheels)
    b.record(vst)
    torch.cuda.synchronize()
    vms, vwall = a.elapsed_time(b) / reps, (time.perf_counter() - t0) * 1e3 / reps
    nv = vd[0] * vd[1] * vd[2]
    out["voxelize"] = {"ms": round(vms, 3), "e2e_ms": round(vwall, 3), "grid": list(vd),
                       "triangles": int(np.asarray(idx).size // 3), "solid_cells": info["solidCells"],
                       "bytes_alg": nv * 24, "achieved_gbs": round(nv * 24 / vms / 1e6, 1),
                       "frac": round(nv * 24 / vms / 1e6 / peak, 4)}
    v.destroy()
    if not no_cpu:
        t0 = time.perf_counter()
        O.voxelize_f64(vd, p, idx, M16)
        out["voxelize"]["cpu_ref_s"] = round(time.perf_counter() - t0, 3)
        out["voxelize"]["cpu_kind"] = "port (f64, the reference's CPU voxelizer)"
        out["voxelize"]["cpu_threads"] = O.threads(0)
    return out


def d2q9_cylinder(peak, no_cpu, updates=4000, chunks=20, launch=None):
    """The D2Q9 cylinder channel (512 x 128, FP32 populations, BGK, D = 20 at (96, 65), u = 0.05,
    Re = 100, rest state with seeded noise): lattice updates per second of the step alone (CUDA
    events around `updates` steps on the solver's stream) and of the reference's sample chunk
    (stepAndSample(50) with its statistics readback, host clock). The two 2.4 MB population
    buffers stay in L2, so the step is bound by launch and synchronisation latency, not by HBM;
    72 B per update (9 populations read and written in FP32) is reported for comparison. `launch`
    (kernel, param, bx, by) replaces the default launch (the persistent kernel, for instance)."""
    import torch

    from windtunnel_vis_b200 import abi as A
    from windtunnel_vis_b200.solver import Solver
    from windtunnel_vis_b200.validation import CHANNEL_DIMS, channel_geometry, channel_params

    dims = CHANNEL_DIMS
    n = dims[0] * dims[1]
    flags, _, sdf = channel_geometry()
    params = channel_params("f32")
    s = Solver(dims, params)
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    if launch is not None:
        s.set_launch(*launch)
    for _ in range(3):
        s.step_and_sample(CHUNK)
    st = torch.cuda.ExternalStream(s.stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(st)
    s.step(updates)
    b.record(st)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / updates
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(chunks):
        s.step_and_sample(CHUNK)
    chunk_s = (time.perf_counter() - t0) / chunks
    used = s.get_launch()
    s.destroy()
    out = {"grid": list(dims), "storage": "f32", "collision": "bgk", "us_per_update": round(ms * 1e3, 3),
           "mlups": round(n / ms / 1e3, 1), "steps_per_s": round(1e3 / ms, 1),
           "chunk_mlups": round(n * CHUNK / chunk_s / 1e6, 1),
           "chunk": f"stepAndSample({CHUNK}) incl. the sampling pass and the statistics readback (host clock)",
           "launch": {"form": "persistent kernel: one cooperative launch per call, work items from an atomic counter, "
                              "grid barrier between steps"}
           if used[0] == A.WT_LAUNCH_PERSISTENT else
           {"form": "10-step CUDA graphs: one launch per step of the persistent kernel's work queue (wall, face "
                    "and bulk items from an atomic counter)"}
           if used[0] == A.WT_LAUNCH_QUEUE else
           {"form": "10-step CUDA graphs: bulk kernel, face rows and wall cells per step",
            "cells_per_thread": used[1], "block": [used[2], used[3]]},
           "bytes_alg_per_update": n * 72, "l2_resident": True,
           "achieved_gbs_equiv": round(n * 72 / ms / 1e6, 1)}
    if not no_cpu:
        from oracle import oracle as O

        o = O.OracleSolver(dims, params)
        o.upload_flags(flags)
        o.upload_sdf(sdf)
        o.step(1)
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < 3.0:
            o.step(20)
            done += 20
        dt = time.perf_counter() - t0
        out["cpu_ref_mlups"] = round(n * done / dt / 1e6, 2)
        out["cpu_threads"] = O.threads(0)
        out["cpu_kind"] = "port"
    return out


def run_reference(args, rank, world):
    """Reference arm: the reference's WGSL path cannot run here (TypeScript + WebGPU; no Node
    and no graphics stack), so its algorithm runs as the CPU restatement on the host cores."""
    if rank != 0:
        return
    n = DIMS[0] * DIMS[1] * DIMS[2]
    from oracle import oracle as O

    th = O.threads(0)
    flags, _, sdf = geometry()
    s = O.OracleSolver(DIMS, PARAMS)
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    for _ in range(max(args.warmup, 0)):
        s.step(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.step(1)
    dt = time.perf_counter() - t0
    v = n * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": list(DIMS), "bench_step": "1 lattice update of the full grid"},
        "cpu_baseline": {"value": round(v, 3), "unit": "MLUPS", "cores": th, "kind": "port",
                         "sample": f"{args.steps} full-grid D3Q19 steps (FP16 storage) on {th} threads"},
        "e2e": {"value": round(v, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank, dist):
    import torch

    from windtunnel_vis_b200.solver import Solver

    torch.cuda.set_device(local_rank)
    flags, frontal, sdf = geometry()
    n = DIMS[0] * DIMS[1] * DIMS[2]
    s = Solver(DIMS, PARAMS)
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    stream = torch.cuda.ExternalStream(s.stream)

    def barrier():
        if dist is not None:
            dist.barrier()

    if args.launch:
        s.set_launch(*(int(v) for v in args.launch.split(",")))
    if args.closure:
        s.set_closure(bench_closure())
    for _ in range(max(args.warmup, 3)):
        s.step_and_sample(CHUNK)
    # the tuner times the Smagorinsky kernel's launches; the closure kernel has one launch shape
    shape = s.get_launch() if (args.launch or args.closure) else s.autotune(10)
    torch.cuda.synchronize()
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = s.launches
    with Clocks(local_rank) as clk:
        torch.cuda.synchronize()
        barrier()
        with torch.cuda.stream(stream):
            t_start.record(stream)
        for k in range(args.steps):
            # stepAndSample(CHUNK): wt_step_and_sample runs step(CHUNK - TAIL) and then one graph of
            # the last TAIL steps, the last of them with the sampling pass fused; calling the two
            # parts here does the same work and lets the events bracket the plain updates for the
            # roofline. The chunk's statistics are read back through the queued form (the
            # reference's stepAndSample Promise): chunk k's plain updates are queued before the
            # host waits for chunk k - 1's statistics, so the device never waits for the host.
            ev[k][0].record(stream)
            s.step(CHUNK - TAIL)
            ev[k][1].record(stream)
            if k > 0:
                s.sample_wait()
            s.step_and_sample_async(TAIL)
        s.sample_wait()
        t_end.record(stream)
        torch.cuda.synchronize()
        barrier()
    launches = s.launches - launches0
    ms = t_start.elapsed_time(t_end)
    sc_ms = sum(a.elapsed_time(b) for a, b in ev) / (args.steps * (CHUNK - TAIL))
    ms_max = max_over_ranks(dist, ms)
    value = replica_mlups(world, n, CHUNK * args.steps, ms_max)

    # end to end through the public API with host buffers, queued the way the reference's app
    # drives its solver (writeBuffer uploads, a stepAndSample promise, mapAsync readbacks): every
    # bench step uploads the body's flags and wall distances from pinned memory and reads the
    # velocity field back; the upload of step k + 1 runs during step k's chunk and the readback of
    # step k during step k + 1's chunk, on the handle's two copy streams. The clock stops after
    # the last readback has landed.
    fl_h = torch.from_numpy(flags).pin_memory()
    sd_h = torch.from_numpy(sdf).pin_memory()
    vel_h = [torch.empty((n, 4), dtype=torch.float16).pin_memory() for _ in range(2)]
    vel_bytes = n * 8
    e2e_steps = max(2, args.steps)
    s.step_and_sample(CHUNK)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    s.upload_flags_async(fl_h.numpy())
    s.upload_sdf_async(sd_h.numpy())
    s.step_and_sample_async(CHUNK)
    for k in range(e2e_steps):
        if k + 1 < e2e_steps:
            s.upload_flags_async(fl_h.numpy())
            s.upload_sdf_async(sd_h.numpy())
        st = s.sample_wait()
        s.read_velocity_half_async(vel_h[k % 2].numpy())
        if k + 1 < e2e_steps:
            s.step_and_sample_async(CHUNK)
    s.sync()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(dist, e2e_s)
    e2e = replica_mlups(world, n, CHUNK * e2e_steps, e2e_s * 1e3)

    if rank != 0:
        s.destroy()
        return
    peak, peak_kind = peaks()
    achieved = n * BYTES_PER_UPDATE / (sc_ms / 1e3) / 1e9
    traffic = measured_traffic(shape, args.closure)
    comps = None
    if world == 1 and not args.no_components and not args.closure:
        comps = components(s, peak, args.no_cpu)
    cpu = None
    if world == 1 and not args.no_cpu:
        mlups, th, done = cpu_port_mlups(args.cpu_seconds)
        cpu = {"value": round(mlups, 3), "unit": "MLUPS", "cores": th, "kind": "port",
               "sample": f"{done} full-grid D3Q19 steps (FP16 storage) of the same workload, ~{args.cpu_seconds:.0f} s"}
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD + (", learned closure in place of Smagorinsky" if args.closure else ""),
                   "grid": list(DIMS), "storage": "f16 shifted (f - w)",
                   "bench_step": f"stepAndSample({CHUNK}): {CHUNK} lattice updates, the last one with the sampling "
                                 "pass fused (velocity field, EMA, sums), the wall force, the 80-byte stats readback",
                   "fused_samples": s.fused_samples,
                   "parallelism": f"replicas{world}", "l2": "inputs larger than L2: 2 x 159 MB population buffers",
                   "launch": {"hint": shape[0], "cells_per_thread": shape[1], "block": [shape[2], shape[3]]}},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": ("one lattice update: k_stream_collide_lc<StF16> (bulk, network on tcgen05) overlapped "
                                "with the face rows and wall cells (features, k_closure_rows on tcgen05, collision)"
                                if args.closure else
                                "one lattice update: k_stream_collide_rows<StF16> (bulk, row pipeline) overlapped "
                                "with k_face_v and k_boundary_tab" if shape[0] == 8 else
                                "k_steps_persistent<D3Q19,StF16>: the chunk's updates in one cooperative launch "
                                "(wall, face and bulk items per step, grid barrier between steps)" if shape[0] == 9 else
                                "one lattice update: k_stream_collide_v<D3Q19,StF16> (bulk) overlapped with "
                                "k_face_v and k_boundary_tab" if shape[1] > 1 else "k_stream_collide<D3Q19,StF16>"),
                     "bytes_alg_per_update": n * BYTES_PER_UPDATE, "traffic_per": "lattice update (ncu, steady state)",
                     "update_ms": round(sc_ms, 5)},
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e, 1), "unit": "MLUPS", "form": "queued calls, copies overlapping the chunks",
                "h2d_bytes_per_step": n * 8,
                "d2h_bytes_per_step": 64 + vel_bytes},
        "gpu_launches": launches,
        "components": comps,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    s.destroy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-components", action="store_true", help="skip the sample / tracer / voxelizer timings")
    ap.add_argument("--launch", default="", help="fixed stream-collide launch 'hint,cells,bx,by' instead of the tuner")
    ap.add_argument("--closure", action="store_true", help="time the step with the learned closure in place of "
                    "Smagorinsky (a seeded network; no component timings)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        run_ours(args, rank, world, local_rank, dist)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
