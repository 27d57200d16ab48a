"""Host-side mirror of the reference's solver interface, over the C ABI of libwt.so.

    LbmSolver / SolverFactory ... src/backend/types.ts:7-18   -> Solver / solver_factory
    Backend ..................... src/backend/types.ts:24-53  -> Backend
    SolverGPU extras ............ src/solver/SolverGPU.ts     -> Solver.read_* / set_wheels / ...
    VoxelizerGPU.voxelize ....... src/voxelize/VoxelizerGPU.ts:48-151 -> Solver.voxelize

Method names are the reference's in snake_case (uploadFlags -> upload_flags, stepAndSample ->
step_and_sample); parameters are the reference's SolverParams dict (u, nu, cs, ground, sides,
spongeNu, spongeStart, spongeIn, tauWall, precision, interp, collision, emaAlpha) and stats come
back as the SolverStats dict (fx, fy, fz, maxU, rhoRef, unstable, step). Errors raise WtError
with the library's message. Every call runs on the GPU through libwt.so; there is no CPU path.
"""
import ctypes as C
import math

import numpy as np

from . import abi

POP_DTYPE = {0: np.float32, 1: np.float16, 2: np.float64}


class WtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{abi.load().wt_error_string(code).decode()} ({code}): {msg}")
        self.code = code


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _stats_dict(st: abi.Stats):
    return {
        "fx": st.fx, "fy": st.fy, "fz": st.fz, "maxU": st.max_u, "rhoRef": st.rho_ref,
        "unstable": bool(st.unstable), "step": int(st.step), "raw": np.array(st.raw[:], np.float64),
        "mass": float(st.mass), "fluidCells": int(st.fluid_cells),
    }


class Solver:
    """One wind tunnel on the current CUDA device (LbmSolver + the SolverGPU extras)."""

    def __init__(self, dims, params: dict):
        self._lib = abi.load()
        self.dims = tuple(int(v) for v in dims)
        nx, ny, nz = self.dims
        self.n = nx * ny * nz
        self.is3d = nz > 1
        self.q = 19 if self.is3d else 9
        self.params = dict(params)
        self.precision = abi.PRECISION[self.params.get("precision", "f32") or "f32"]
        # host arrays of queued copies, kept referenced until the library is done with them: uploads
        # until the next step or sample has applied them, readbacks until a later sample has waited
        # for them (or sync / destroy)
        self._up_refs, self._rd_refs, self._rd_before_sample = [], [], 0
        h = C.c_void_p()
        d = abi.Dims(nx, ny, nz)
        rc = self._lib.wt_create(C.byref(d), C.byref(abi.make_params(self.params)), C.byref(h))
        if rc != 0:
            raise WtError(rc, self._lib.wt_last_error(None).decode())
        self._h = h

    # ---- plumbing ----------------------------------------------------------------------------
    def _check(self, rc):
        if rc != 0:
            raise WtError(rc, self._lib.wt_last_error(self._h).decode())

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        """cudaStream_t of this tunnel (for torch.cuda.ExternalStream event timing)."""
        return int(self._lib.wt_stream(self._h) or 0)

    @property
    def device(self) -> int:
        return int(self._lib.wt_device(self._h))

    @property
    def launches(self) -> int:
        return int(self._lib.wt_launch_count(self._h))

    @property
    def fused_samples(self) -> int:
        """stepAndSample calls whose last step ran the sampling pass fused (wt_fused_sample_count)."""
        return int(self._lib.wt_fused_sample_count(self._h))

    @property
    def step_count(self) -> int:
        return int(self._lib.wt_step_count(self._h))

    def destroy(self):
        if getattr(self, "_h", None):
            self._lib.wt_destroy(self._h)  # waits for the queued copies first
            self._h = None
        self._up_refs, self._rd_refs, self._rd_before_sample = [], [], 0

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # ---- parameters --------------------------------------------------------------------------
    def set_params(self, p: dict):
        self.params.update(p)
        self._check(self._lib.wt_set_params(self._h, C.byref(abi.make_params(self.params))))

    def kparams(self) -> abi.KParams:
        k = abi.KParams()
        self._check(self._lib.wt_get_kparams(self._h, C.byref(k)))
        return k

    def reset(self):
        self._check(self._lib.wt_reset(self._h))

    def clear_stats(self):
        self._check(self._lib.wt_clear_stats(self._h))

    # ---- learned closure (wt_set_closure) -----------------------------------------------------
    def set_closure(self, model):
        """Installs the learned closure (a dict of arrays, see windtunnel_vis_b200.closure, or an
        abi.Closure) in place of Smagorinsky; None restores Smagorinsky."""
        if model is None:
            self._check(self._lib.wt_set_closure(self._h, None))
            return
        from .closure import to_struct

        c = model if isinstance(model, abi.Closure) else to_struct(model)
        self._check(self._lib.wt_set_closure(self._h, C.byref(c)))

    def get_closure(self):
        c = abi.Closure()
        on = C.c_int32()
        self._check(self._lib.wt_get_closure(self._h, C.byref(c), C.byref(on)))
        if not on.value:
            return None
        from .closure import from_struct

        return from_struct(c)

    # ---- geometry ----------------------------------------------------------------------------
    def upload_flags(self, flags):
        f = np.ascontiguousarray(np.asarray(flags).ravel(), np.uint32)
        self._check(self._lib.wt_upload_flags(self._h, _ptr(f), f.size))

    def upload_sdf(self, d):
        a = np.ascontiguousarray(np.asarray(d).ravel(), np.float32)
        self._check(self._lib.wt_upload_sdf(self._h, _ptr(a), a.size))

    def upload_flags_async(self, flags):
        """uploadFlags queued (device.queue.writeBuffer): the copy overlaps the work in flight and
        the geometry applies to every later call. The array (kept referenced here until `sync`)
        must not change until the next call that reads the geometry; page-locked memory (e.g. a
        pinned torch tensor's numpy view) lets the copy overlap."""
        f = np.ascontiguousarray(np.asarray(flags).ravel(), np.uint32)
        self._check(self._lib.wt_upload_flags_async(self._h, _ptr(f), f.size))
        self._up_refs.append(f)

    def upload_sdf_async(self, d):
        """uploadSdf queued, as `upload_flags_async`."""
        a = np.ascontiguousarray(np.asarray(d).ravel(), np.float32)
        self._check(self._lib.wt_upload_sdf_async(self._h, _ptr(a), a.size))
        self._up_refs.append(a)

    def set_wheels(self, wheels):
        arr, n = abi.make_wheels(list(wheels))
        self._check(self._lib.wt_set_wheels(self._h, arr, n))

    def voxelize(self, positions, indices, matrix, wheels=()):
        """Backend.voxelize / VoxelizerGPU.voxelize: mesh (f32 xyz, u32 indices), column-major
        4x4 mesh->grid matrix, grid-space wheels -> VoxelInfo dict."""
        pos = np.ascontiguousarray(np.asarray(positions).ravel(), np.float32)
        idx = np.ascontiguousarray(np.asarray(indices).ravel(), np.uint32)
        m = np.ascontiguousarray(np.asarray(matrix, np.float64).ravel(), np.float32)
        if m.size != 16:
            raise ValueError("matrix must have 16 elements (column-major 4x4)")
        arr, nw = abi.make_wheels(list(wheels))
        info = abi.VoxelInfo()
        self._check(self._lib.wt_voxelize(self._h, _ptr(pos), pos.size // 3, _ptr(idx), idx.size // 3, _ptr(m), arr,
                                          nw, C.byref(info)))
        return {"frontal": info.frontal, "solidCells": info.solid_cells, "min": list(info.min), "max": list(info.max)}

    # ---- stepping ----------------------------------------------------------------------------
    def step(self, steps: int):
        self._check(self._lib.wt_step(self._h, int(steps)))

    def sample(self):
        st = abi.Stats()
        self._check(self._lib.wt_sample(self._h, C.byref(st)))
        return _stats_dict(st)

    def step_and_sample(self, steps: int):
        st = abi.Stats()
        self._check(self._lib.wt_step_and_sample(self._h, int(steps), C.byref(st)))
        return _stats_dict(st)

    def step_and_sample_async(self, steps: int):
        """stepAndSample in the reference's asynchronous form: queues the chunk and returns; the
        statistics come from `sample_wait`."""
        self._check(self._lib.wt_step_and_sample_async(self._h, int(steps)))
        self._up_refs.clear()  # applied before the chunk was queued
        # the chunk's sampling step waits for every readback queued before it
        self._rd_before_sample = len(self._rd_refs)

    def sample_wait(self):
        st = abi.Stats()
        self._check(self._lib.wt_sample_wait(self._h, C.byref(st)))
        del self._rd_refs[:self._rd_before_sample]
        self._rd_before_sample = 0
        return _stats_dict(st)

    def sync(self):
        """Waits for every queued step, sample, upload and readback of the handle."""
        self._check(self._lib.wt_sync(self._h))
        self._up_refs.clear()
        self._rd_refs.clear()
        self._rd_before_sample = 0

    # ---- readback / checkpoint ---------------------------------------------------------------
    def read_flags(self):
        out = np.empty(self.n, np.uint32)
        self._check(self._lib.wt_read_flags(self._h, _ptr(out), self.n))
        return out

    def read_sdf_encoded(self):
        out = np.empty(self.n, np.uint32)
        self._check(self._lib.wt_read_sdf(self._h, _ptr(out), self.n))
        return out

    def read_populations(self):
        """Raw current buffer: float32 / float16 (f - w) / float64, shape (q * n,)."""
        out = np.empty(self.q * self.n, POP_DTYPE[self.precision])
        self._check(self._lib.wt_read_populations(self._h, _ptr(out), out.nbytes))
        return out

    def write_populations(self, a):
        a = np.ascontiguousarray(a, POP_DTYPE[self.precision]).ravel()
        self._check(self._lib.wt_write_populations(self._h, _ptr(a), a.nbytes))

    def read_velocity(self, out=None):
        """(ux, uy, uz, rho) per cell as float32, shape (n, 4): the velocity texture the renderer
        samples. `out` (optional) is a C-contiguous float32 array of that shape to fill, e.g. a
        view of pinned host memory."""
        if out is None:
            out = np.empty((self.n, 4), np.float32)
        elif out.dtype != np.float32 or out.size != 4 * self.n or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of n x 4 values")
        self._check(self._lib.wt_read_velocity(self._h, _ptr(out), self.n))
        return out

    def read_velocity_half(self, out=None):
        """The velocity field in its storage format: (n, 4) float16 (ux, uy, uz, rho), the
        reference's rgba16float texture. `out` (optional): a C-contiguous float16 array of that
        shape, e.g. a view of pinned host memory."""
        if out is None:
            out = np.empty((self.n, 4), np.float16)
        assert out.dtype == np.float16 and out.shape == (self.n, 4) and out.flags["C_CONTIGUOUS"]
        self._check(self._lib.wt_read_velocity_half4(self._h, _ptr(out), self.n))
        return out

    def read_velocity_half_async(self, out):
        """`read_velocity_half` queued: the copy into `out` (a C-contiguous (n, 4) float16 array,
        page-locked for the copy to overlap) starts once the work queued so far is done; `out`
        holds the field after `sync`."""
        assert out.dtype == np.float16 and out.shape == (self.n, 4) and out.flags["C_CONTIGUOUS"]
        self._check(self._lib.wt_read_velocity_half4_async(self._h, _ptr(out), self.n))
        self._rd_refs.append(out)
        return out

    def read_means(self):
        a = np.empty((self.n, 4), np.float32)
        b = np.empty(self.n, np.float32)
        self._check(self._lib.wt_read_means(self._h, _ptr(a), _ptr(b), self.n))
        return a, b

    # ---- derived fields / export ---------------------------------------------------------------
    def derive_fields(self):
        """The derived pass: vorticity, Q-criterion, turbulence intensity, binary16 mean field."""
        self._check(self._lib.wt_derive_fields(self._h))

    def read_derived(self):
        """(vort (n, 4) = wx, wy, wz, Q; stat (n, 4) = TI, solid, 0, 0; mean (n, 4)) as float32."""
        out = [np.empty((self.n, 4), np.float32) for _ in range(3)]
        self._check(self._lib.wt_read_derived(self._h, *(_ptr(a) for a in out), self.n))
        return tuple(out)

    def export_fields(self, stride: int):
        """SolverGPU.exportFields: FieldExport dict {dims, stride, vel, mean, vort}, every field a
        float32 array of shape (points, 4), x fastest."""
        stride = int(stride)
        o = [-(-d // stride) for d in self.dims]
        n = o[0] * o[1] * o[2]
        vel, mean, vort = (np.empty((n, 4), np.float32) for _ in range(3))
        self._check(self._lib.wt_export_fields(self._h, stride, _ptr(vel), _ptr(mean), _ptr(vort), n))
        return {"dims": tuple(o), "stride": stride, "vel": vel, "mean": mean, "vort": vort}

    def streamlines(self, sp: abi.StreamlineParams):
        """The streamline pass: (seeds * points, 4) float32 (x, y, z, speed; -1 after the end)."""
        out = np.empty((sp.seeds * sp.points, 4), np.float32)
        self._check(self._lib.wt_streamlines(self._h, C.byref(sp), _ptr(out), out.shape[0]))
        return out

    def probes(self, positions):
        """Backend.probeData: per probe {'inst': [ux, uy, uz, rho], 'mean': [...]} (at most 8)."""
        pos = np.zeros((len(positions), 4), np.float32)
        for k, p in enumerate(positions):
            pos[k, :3] = p[:3]
        out = np.empty((len(positions), 8), np.float32)
        self._check(self._lib.wt_probes(self._h, _ptr(pos), len(positions), _ptr(out)))
        return [{"inst": out[k, :4].tolist(), "mean": out[k, 4:].tolist()} for k in range(len(positions))]

    # ---- launch shape ------------------------------------------------------------------------
    def set_launch(self, kernel, param, bx=0, by=0):
        """Stream-collide launch: kernel = occupancy hint (0 none, 2..4 CTAs of 256 threads per
        SM), param = cells per thread along x (1 = the scalar kernel, 2 or 4), block bx x by
        (0 = default). kernel = 8 (param 2, bx 0) selects the row pipeline with `by` interior rows
        per block (0 = 4); kernel = 9 (param 2, bx 0, by 0) the persistent kernel, which takes all
        the steps of a call in one launch."""
        self._check(self._lib.wt_set_launch(self._h, int(kernel), int(param), int(bx), int(by)))

    def get_launch(self):
        out = (C.c_int32 * 4)()
        self._check(self._lib.wt_get_launch(self._h, out))
        return tuple(out)

    def set_wait_limit(self, polls):
        """Test hook: polls of each row-pipeline consumer wait before it gives up (negative: the
        default)."""
        self._check(self._lib.wt_set_wait_limit(self._h, int(polls)))

    def autotune(self, iters=20):
        """The launch tuner: returns the chosen (kernel, param, bx, by)."""
        out = (C.c_int32 * 4)()
        self._check(self._lib.wt_autotune(self._h, int(iters), out))
        return tuple(out)

    # ---- tracers -----------------------------------------------------------------------------
    def advect_tracers(self, tp: abi.TracerParams):
        self._check(self._lib.wt_advect_tracers(self._h, C.byref(tp)))

    def read_tracers(self, count, trail):
        s = np.empty((count, 4), np.float32)
        h = np.empty((count * trail, 4), np.float32)
        self._check(self._lib.wt_read_tracers(self._h, _ptr(s), count, _ptr(h), count * trail))
        return s, h

    def write_tracers(self, state, hist, trail):
        s = np.ascontiguousarray(state, np.float32).reshape(-1, 4)
        h = np.ascontiguousarray(hist, np.float32).reshape(-1, 4)
        self._check(self._lib.wt_write_tracers(self._h, _ptr(s), s.shape[0], _ptr(h), h.shape[0], int(trail)))


class Batch:
    """Many independent tunnels stepped together (wt_batch): pairs of steps replay one CUDA graph
    holding every member's step kernels, so small tunnels run concurrently. Members stay ordinary
    Solver objects for parameters, geometry and readback, and must outlive the batch."""

    def __init__(self, solvers, fused=False, persistent=False, queue=False):
        self._lib = abi.load()
        self.members = list(solvers)
        arr = (C.c_void_p * len(self.members))(*[s.handle.value for s in self.members])
        h = C.c_void_p()
        rc = self._lib.wt_batch_create(arr, len(self.members), C.byref(h))
        if rc != 0:
            raise WtError(rc, self._lib.wt_last_error(None).decode())
        self._h = h
        if fused:
            self.set_fused(True)
        if persistent:
            self.set_persistent(True)
        if queue:
            self.set_queue(True)

    def set_fused(self, on: bool):
        """Bulk rows of all members in one batch-kernel launch per step (wt_batch_set_fused(b, 1))."""
        self._check(self._lib.wt_batch_set_fused(self._h, 1 if on else 0))

    def set_persistent(self, on: bool):
        """Every wt_batch_step call of two or more steps as one cooperative launch of the
        persistent kernel over all members (wt_batch_set_fused(b, WT_BATCH_PERSISTENT))."""
        self._check(self._lib.wt_batch_set_fused(self._h, abi.WT_BATCH_PERSISTENT if on else 0))

    def set_queue(self, on: bool):
        """Every step of every member as one launch of the persistent kernel's work queue, the
        launches captured in the batch graphs (wt_batch_set_fused(b, WT_BATCH_QUEUE))."""
        self._check(self._lib.wt_batch_set_fused(self._h, abi.WT_BATCH_QUEUE if on else 0))

    def _check(self, rc):
        if rc != 0:
            raise WtError(rc, self._lib.wt_batch_last_error(self._h).decode())

    def step(self, steps: int):
        self._check(self._lib.wt_batch_step(self._h, int(steps)))

    def sample(self):
        out = (abi.Stats * len(self.members))()
        self._check(self._lib.wt_batch_sample(self._h, out))
        return [_stats_dict(out[k]) for k in range(len(self.members))]

    def step_and_sample(self, steps: int):
        self.step(steps)
        return self.sample()

    def destroy(self):
        if getattr(self, "_h", None):
            self._lib.wt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def solver_factory(dims, params: dict) -> Solver:
    """SolverFactory (src/backend/types.ts:18)."""
    return Solver(dims, params)


def pack_params(dims, params: dict) -> abi.KParams:
    """SolverGPU.writeParams (src/solver/SolverGPU.ts:160-187) through the library."""
    k = abi.KParams()
    nx, ny, nz = dims
    rc = abi.load().wt_pack_params(C.byref(abi.Dims(nx, ny, nz)), C.byref(abi.make_params(params)), C.byref(k))
    if rc != 0:
        raise WtError(rc, "wt_pack_params")
    return k


def fits(dims, precision="f32"):
    """Backend.fits (src/backend/webgpu.ts:58-61): (fits, bytes_needed) on the current device."""
    nx, ny, nz = dims
    need = C.c_int64()
    ok = C.c_int32()
    rc = abi.load().wt_fits(C.byref(abi.Dims(nx, ny, nz)), abi.PRECISION[precision], C.byref(need), C.byref(ok))
    if rc != 0:
        raise WtError(rc, abi.load().wt_last_error(None).decode())
    return bool(ok.value), int(need.value)


class Backend:
    """Compute half of the reference's Backend (src/backend/types.ts:24-53): owns one solver and
    runs frames of `steps` steps with a statistics sample, plus voxelization and tracers.
    Rendering members of the reference (canvas, pixelSize, draw) have no counterpart here."""

    kind = "cuda"
    supports3D = True

    def __init__(self):
        self.solver = None
        self.particles = None

    @property
    def label(self):
        return "CUDA sm_100a"

    @property
    def step_count(self):
        return self.solver.step_count if self.solver else 0

    @property
    def cells(self):
        return self.solver.n if self.solver else 0

    def fits(self, dims, precision="f32"):
        return fits(dims, precision)[0]

    def create_solver(self, dims, params: dict):
        if self.solver:
            self.solver.destroy()
        self.solver = Solver(dims, params)
        return self.solver

    def set_params(self, p: dict):
        self.solver.set_params(p)

    def reset(self):
        self.solver.reset()

    def clear_stats(self):
        self.solver.clear_stats()

    def voxelize(self, positions, indices, matrix, wheels=()):
        return self.solver.voxelize(positions, indices, matrix, wheels)

    def frame(self, steps, on_stats=None, tracers: abi.TracerParams = None):
        """`steps` solver steps, the macro / statistics pass, and (optionally) one tracer
        dispatch against the fresh velocity field. Returns SolverStats."""
        st = self.solver.step_and_sample(steps)
        if tracers is not None:
            self.solver.advect_tracers(tracers)
        if on_stats:
            on_stats(st)
        return st

    def export_fields(self, max_points: int):
        """Backend.exportFields (src/backend/webgpu.ts:133-137): the stride that keeps the point
        count at or below about max_points, then SolverGPU.exportFields."""
        stride = max(1, math.ceil(float(np.cbrt(self.solver.n / max_points))))
        return self.solver.export_fields(stride)

    def probe_data(self, positions):
        """Backend.probeData: instantaneous and mean samples at up to 8 probe points."""
        return self.solver.probes(positions)

    def solver_factory(self):
        return solver_factory

    def destroy(self):
        if self.solver:
            self.solver.destroy()
            self.solver = None
