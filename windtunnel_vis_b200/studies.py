"""Host-side consumer of the solver: the app's flow / statistics loop with its stability watchdog,
and the studies panel's pinned results and parameter sweeps.

Tunnel ..... the reference App's flow mapping, convective clock, coefficient averaging and
             watchdog (src/app.ts:319-442): updateFlow / resetFlow, handleInstability (lattice
             speed x0.85 while above 0.55 of nominal, else viscosity x1.6; viscosity x1.25 in
             both cases; restart from the initial state), onStats (stale samples dropped, local
             Mach above 0.6 or an unstable sample triggers the watchdog at most once per 30
             frames, start-up transients kept out of the averages), statsSince / readout.
Studies .... pinned results, CSV table and parameter sweeps (src/ui/studies.ts:7-253): each point
             applies one parameter (speed, yaw, pitch or ride height), lets the flow settle for
             `settle` convective times and averages the coefficients over the next `avg`.

Rendering, thumbnails and widgets of the reference have no counterpart here.
"""
import math

from . import mesh as Mh
from .analysis import Ema, coefficients, drag_newtons, map_flow, window_stats
from .export import csv
from .solver import Backend

AVG_WINDOW = 4.0  # convective times of the readout window
V_MAX_KMH = 300.0
CFG_KEYS = ("vehicle", "lengthM", "yaw", "pitch", "rideMm", "speedKmh", "nuAir", "reOverrideOn", "reOverride",
            "ground", "lesCs")
SWEEP_PARAMS = {
    "yaw": {"label": "Yaw (crosswind)", "unit": "°", "from": 0.0, "to": 15.0, "n": 4},
    "speedKmh": {"label": "Wind speed", "unit": "km/h", "from": 60.0, "to": 240.0, "n": 4},
    "rideMm": {"label": "Ride height offset", "unit": "mm", "from": 0.0, "to": 150.0, "n": 4},
    "pitch": {"label": "Pitch", "unit": "°", "from": -3.0, "to": 3.0, "n": 4},
}


class Series:
    def __init__(self):
        self.t, self.v = [], []

    def push(self, t, v):
        self.t.append(t)
        self.v.append(v)

    def clear(self):
        self.t.clear()
        self.v.clear()


class Tunnel:
    """One vehicle in a tunnel on the CUDA backend, driven frame by frame like the reference app.

    mesh: dict(positions, indices, wheels (normalised space), min, max, name) as from
    mesh.vehicle_body / mesh.normalize_mesh; settings: the reference's state fields used here."""

    def __init__(self, dims, mesh, settings=None, precision="f16", steps_per_frame=50, backend=None):
        self.dims = tuple(dims)
        self.is3d = self.dims[2] > 1
        self.mesh = mesh
        self.s = dict(vehicle=mesh.get("name", "vehicle"), lengthM=4.8, yaw=0.0, pitch=0.0, rideMm=0.0,
                      speedKmh=120.0, nuAir=1.5, reOverrideOn=False, reOverride=0.0, ground="moving", lesCs=0.14,
                      rotatingWheels=True, lengthFrac=1 / 3, xFrac=0.34)
        self.s.update(settings or {})
        self.precision = precision
        self.steps_per_frame = steps_per_frame
        self.backend = backend if backend is not None else Backend()
        self.stab = {"uScale": 1.0, "nuScale": 1.0, "events": 0}
        self.frames = 0
        self.last_stab_frame = -1000
        self.clock = 0.0
        self.avg_start = 1.0
        self.last_sample_step = 0
        self.cd_avg, self.cl_avg, self.cs_avg = Ema(0.05), Ema(0.05), Ema(0.05)
        self.raw = {"cd": Series(), "cl": Series(), "cs": Series()}
        self.cd_inst = math.nan
        self.last_stats = None
        self.vinfo = {"frontal": 1}
        self.l_cells = 100.0
        self.update_flow()
        self.cur = {"U": self.flow["U"], "nu": self.flow["nu"]}
        self.backend.create_solver(self.dims, self._params())
        self.revoxelize()

    # ---- flow mapping (app.ts:319-349) ------------------------------------------------------------
    def update_flow(self):
        s = self.s
        self.flow = map_flow(s["speedKmh"] / 3.6, s["lengthM"], s["nuAir"] * 1e-5, self.l_cells, V_MAX_KMH / 3.6,
                             0.0006 if self.is3d else 0.0003, s["reOverride"] if s["reOverrideOn"] else None,
                             self.stab["uScale"], self.stab["nuScale"])

    def _params(self):
        return dict(u=self.cur["U"], nu=self.cur["nu"], cs=self.s["lesCs"], ground=self.s["ground"],
                    sides="freeslip", spongeNu=0.03, spongeStart=0.85, emaAlpha=0.0, precision=self.precision)

    def reset_flow(self):
        self.cur = {"U": self.flow["U"], "nu": self.flow["nu"]}
        self.backend.set_params(self._params())
        self.backend.reset()
        self.clock = 0.0
        self.avg_start = 1.0
        self.last_sample_step = 0
        for e in (self.cd_avg, self.cl_avg, self.cs_avg):
            e.reset()
        for r in self.raw.values():
            r.clear()

    def flow_changed(self):
        self.update_flow()
        self.reset_flow()

    def revoxelize(self):
        """Place the body (yaw, pitch, ride height) and voxelize it (app.ts:270-300)."""
        s = self.s
        m = self.mesh
        dx_real = s["lengthM"] / (s["lengthFrac"] * self.dims[0])
        pl = dict(mode="ground", lengthFrac=s["lengthFrac"], diamFrac=0.3, xFrac=s["xFrac"], yawDeg=s["yaw"],
                  pitchDeg=s["pitch"], rideCells=s["rideMm"] / 1000.0 / dx_real)
        M16, scale, full = Mh.placement_matrix(m["positions"], m["min"], m["max"], self.dims, pl)
        self.l_cells = scale
        wheels = Mh.grid_wheels(m.get("wheels", []), full) if (s["rotatingWheels"] and self.is3d) else []
        self.vinfo = self.backend.voxelize(m["positions"], m["indices"], M16, wheels)
        self.update_flow()
        self.reset_flow()

    # ---- watchdog and statistics (app.ts:366-420) --------------------------------------------------
    def handle_instability(self, reason):
        self.last_stab_frame = self.frames
        self.stab["events"] += 1
        if self.stab["uScale"] > 0.55:
            self.stab["uScale"] *= 0.85
        else:
            self.stab["nuScale"] *= 1.6
        self.stab["nuScale"] *= 1.25
        self.update_flow()
        self.reset_flow()
        return reason

    def on_stats(self, st):
        if st["step"] == 0 or st["step"] > self.backend.step_count:
            return None
        self.last_stats = st
        mach = st["maxU"] * math.sqrt(3.0)
        if (st["unstable"] or mach > 0.6) and self.frames - self.last_stab_frame < 30:
            return None
        if st["unstable"]:
            return self.handle_instability(f"Ma = {mach:.2f}" if math.isfinite(st["fx"]) else "NaN")
        if mach > 0.6:
            return self.handle_instability(f"local Mach {mach:.2f} > 0.6")
        U = self.cur["U"]
        c = coefficients(st["fx"], st["fy"], st["fz"], U, max(self.vinfo["frontal"], 1), st["rhoRef"])
        t_conv = self.clock - max(0, self.backend.step_count - st["step"]) * U / self.l_cells
        dt = st["step"] - self.last_sample_step if self.last_sample_step else 0
        self.last_sample_step = st["step"]
        k = 1.0 - math.exp(-(dt * U) / (1.5 * self.l_cells)) if dt > 0 else 0.05
        for e in (self.cd_avg, self.cl_avg, self.cs_avg):
            e.k = min(max(k, 0.002), 1.0)
        self.cd_inst = c["cd"]
        if t_conv < self.avg_start:
            return None
        self.cd_avg.push(c["cd"])
        self.cl_avg.push(c["cl"])
        self.cs_avg.push(c["cs"])
        for key in ("cd", "cl", "cs"):
            self.raw[key].push(t_conv, c[key])
        return None

    def frame(self):
        """One frame: steps, sample, convective clock, statistics. Returns the watchdog's reason
        when it restarted the flow, else None."""
        st = self.backend.frame(self.steps_per_frame)
        self.frames += 1
        self.clock += self.steps_per_frame * self.cur["U"] / self.l_cells
        return self.on_stats(st)

    def stats_since(self, t0):
        def w(s):
            return window_stats(s.t, s.v, max(0.0, (s.t[-1] if s.t else 0.0) - t0))
        return {k: w(self.raw[k]) for k in ("cd", "cl", "cs")}

    def readout(self):
        w = {k: window_stats(self.raw[k].t, self.raw[k].v, AVG_WINDOW) for k in ("cd", "cl", "cs")}

        def pick(st, ema):
            return st["mean"] if math.isfinite(st["mean"]) else ema.value

        sd = w["cd"]
        cd = pick(sd, self.cd_avg)
        d = self.dims
        blockage = self.vinfo["frontal"] / (d[1] * d[2] if self.is3d else d[1])
        dx = self.flow["dx"]
        frontal_m2 = self.vinfo["frontal"] * dx * dx
        converged = sd["span"] >= AVG_WINDOW * 0.75 and math.isfinite(sd["se"]) and \
            sd["se"] < max(0.02 * abs(sd["mean"]), 0.005)
        return {"cd": cd, "cl": pick(w["cl"], self.cl_avg), "cs": pick(w["cs"], self.cs_avg), "cdInst": self.cd_inst,
                "cdSE": sd["se"], "avgSpan": sd["span"], "converged": converged,
                "cdCorrected": cd * (1 - blockage) ** 2, "frontalM2": frontal_m2,
                "dragN": drag_newtons(cd, self.s["speedKmh"] / 3.6, frontal_m2), "flow": self.flow,
                "convTime": self.clock, "maxMach": self.last_stats["maxU"] * math.sqrt(3) if self.last_stats else 0.0,
                "blockage": blockage}

    def destroy(self):
        self.backend.destroy()


class Studies:
    """Pinned results and parameter sweeps over a Tunnel (src/ui/studies.ts)."""

    def __init__(self, tunnel: Tunnel):
        self.t = tunnel
        self.pinned = []
        self.sweep = None

    def cfg(self):
        return {k: self.t.s.get(k) for k in CFG_KEYS}

    def describe(self, cfg):
        bits = [str(cfg["vehicle"]), f"{cfg['speedKmh']:.0f} km/h"]
        if cfg["yaw"]:
            bits.append(f"yaw {cfg['yaw']:.1f}°")
        if cfg["pitch"]:
            bits.append(f"pitch {cfg['pitch']:.1f}°")
        if cfg["rideMm"]:
            bits.append(f"ride +{cfg['rideMm']:.0f} mm")
        bits.append("3D" if self.t.is3d else "2D")
        return " · ".join(bits)

    def pin_current(self, label=None):
        r = self.t.readout()
        if not math.isfinite(r["cd"]):
            return None
        cfg = self.cfg()
        p = {"label": label or self.describe(cfg), "cfg": cfg, "cd": r["cd"], "cdSE": r["cdSE"], "cl": r["cl"],
             "cs": r["cs"], "dragN": r["dragN"], "converged": r["converged"], "reSim": r["flow"]["reSim"]}
        self.pinned.append(p)
        return p

    def export_csv(self):
        rows = [[p["label"], p["cd"], p["cdSE"], p["cl"], p["cs"], p["dragN"], p["reSim"],
                 "true" if p["converged"] else "false", *[str(p["cfg"][k]).lower() if isinstance(p["cfg"][k], bool)
                                                          else str(p["cfg"][k]) for k in CFG_KEYS]]
                for p in self.pinned]
        return csv(["label", "cd", "cd_se", "cl", "cs", "drag_N", "re_sim", "converged", *CFG_KEYS], rows)

    def apply(self, param, v):
        s = self.t.s
        if param == "speedKmh":
            s["speedKmh"] = v
            self.t.flow_changed()
        else:
            if param == "yaw":
                s["yaw"] = v
            if param == "pitch":
                s["pitch"] = v
            if param == "rideMm":
                s["rideMm"] = max(0.0, v)
            self.t.revoxelize()

    def run_sweep(self, param, values, settle=2.0, avg=3.0, max_frames=1_000_000):
        if param == "yaw" and not self.t.is3d:
            raise ValueError("Yaw sweeps need the 3D solver")
        self.sweep = {"param": param, "pts": []}
        for v in values:
            self.apply(param, v)
            t0 = self.t.clock + settle
            frames = 0
            while self.t.clock < t0 + avg and frames < max_frames:
                self.t.frame()
                frames += 1
            st = self.t.stats_since(t0)
            self.sweep["pts"].append({"v": v, "cd": st["cd"]["mean"], "cdSE": st["cd"]["se"], "cl": st["cl"]["mean"],
                                      "cs": st["cs"]["mean"]})
            self.pin_current(f"{self.describe(self.cfg())} (sweep)")
        return self.sweep


def sweep_values(param, n=None, lo=None, hi=None):
    """The panel's sweep points: N = clamp(round(n), 2, 20) values a + (b - a) i / (N - 1), with
    the parameter's defaults for the fields not given."""
    p = SWEEP_PARAMS[param]
    N = max(2, min(20, int(math.floor((p["n"] if n is None else n) + 0.5))))
    a = p["from"] if lo is None else float(lo)
    b = p["to"] if hi is None else float(hi)
    return [a + ((b - a) * i) / (N - 1) for i in range(N)]
