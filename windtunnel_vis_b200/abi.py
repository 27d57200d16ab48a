"""ctypes mirror of include/wt.h (the C ABI of libwt.so).

Struct layouts here must match include/wt.h field for field; tests/test_abi.py checks sizes and
offsets against the header. Field names follow the reference's SolverParams / SolverStats /
VoxelInfo / WheelDef (src/solver/types.ts, src/voxelize/VoxelizerGPU.ts:6-12, mesh.ts:54-60).
"""
import ctypes as C
import os

WT_OK = 0
WT_E_INVALID = -1
WT_E_CUDA = -2
WT_E_OOM = -3
WT_E_STATE = -4
WT_E_UNSUPPORTED = -5
WT_E_NO_DEVICE = -6
WT_LAUNCH_ROW_PIPELINE = 8
WT_LAUNCH_PERSISTENT = 9
WT_LAUNCH_QUEUE = 10
WT_BATCH_PERSISTENT = 2
WT_BATCH_QUEUE = 3

GROUND = {"freeslip": 0, "noslip": 1, "moving": 2}
SIDES = {"freeslip": 0, "periodic": 1}
PRECISION = {"f32": 0, "f16": 1, "f64": 2}
COLLISION = {"regularized": 0, "bgk": 1}
INIT = {"freestream": 0, "rest_noise": 1}


class Dims(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32)]


class Params(C.Structure):
    _fields_ = [
        ("u", C.c_double), ("nu", C.c_double), ("cs", C.c_double),
        ("sponge_nu", C.c_double), ("sponge_start", C.c_double), ("sponge_in", C.c_double),
        ("tau_wall", C.c_double), ("ema_alpha", C.c_double), ("init_noise", C.c_double),
        ("ground", C.c_int32), ("sides", C.c_int32), ("precision", C.c_int32),
        ("interp", C.c_int32), ("collision", C.c_int32), ("init_mode", C.c_int32),
        ("init_seed", C.c_uint32), ("reserved", C.c_uint32),
    ]


class KParams(C.Structure):
    _fields_ = [
        ("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("n", C.c_uint32),
        ("tau0", C.c_float), ("csmag2", C.c_float), ("uin", C.c_float), ("rho_in", C.c_float),
        ("ground", C.c_uint32), ("stride_x", C.c_uint32), ("sponge_start", C.c_float), ("sponge_nu", C.c_float),
        ("u_ground", C.c_float), ("ema_alpha", C.c_float), ("u_ref", C.c_float), ("ref_x", C.c_uint32),
        ("side_mode", C.c_uint32), ("collision", C.c_uint32), ("tau_wall", C.c_float), ("pad2", C.c_uint32),
        ("sponge_in", C.c_float), ("contact_h", C.c_float), ("interp", C.c_uint32), ("stride_p", C.c_uint32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("fx", C.c_double), ("fy", C.c_double), ("fz", C.c_double),
        ("max_u", C.c_double), ("rho_ref", C.c_double), ("step", C.c_int64),
        ("unstable", C.c_int32), ("reserved", C.c_int32), ("raw", C.c_double * 8),
        ("mass", C.c_double), ("fluid_cells", C.c_int64),
    ]


class Wheel(C.Structure):
    _fields_ = [("c", C.c_double * 3), ("axis", C.c_double * 3), ("r", C.c_double), ("hw", C.c_double)]


class VoxelInfo(C.Structure):
    _fields_ = [("frontal", C.c_int32), ("solid_cells", C.c_int32), ("min", C.c_int32 * 3), ("max", C.c_int32 * 3)]


class TracerParams(C.Structure):
    _fields_ = [
        ("count", C.c_uint32), ("trail", C.c_uint32), ("head", C.c_uint32), ("emitter", C.c_uint32),
        ("steps", C.c_float), ("seed", C.c_uint32), ("max_age", C.c_float), ("nozzles", C.c_uint32),
        ("rake_a", C.c_float * 4), ("rake_b", C.c_float * 4),
        ("advance", C.c_uint32), ("fill", C.c_uint32), ("lines", C.c_uint32), ("pad", C.c_uint32),
        ("rake_d", C.c_float * 4),
    ]


class StreamlineParams(C.Structure):
    _fields_ = [
        ("seeds", C.c_uint32), ("points", C.c_uint32), ("use_mean", C.c_uint32), ("per_line", C.c_uint32),
        ("rake_a", C.c_float * 4), ("rake_b", C.c_float * 4),
        ("h", C.c_float), ("p0", C.c_float), ("p1", C.c_float), ("p2", C.c_float),
        ("rake_d", C.c_float * 4),
    ]


CLOSURE_IN = 10
CLOSURE_HID = 32


class Closure(C.Structure):
    """wt_closure: feature normalisation, the 10 -> 32 -> 32 -> 1 network, output scale."""
    _fields_ = [
        ("shift", C.c_float * CLOSURE_IN), ("scale", C.c_float * CLOSURE_IN),
        ("w1", (C.c_float * CLOSURE_HID) * CLOSURE_IN), ("b1", C.c_float * CLOSURE_HID),
        ("w2", (C.c_float * CLOSURE_HID) * CLOSURE_HID), ("b2", C.c_float * CLOSURE_HID),
        ("w3", C.c_float * CLOSURE_HID), ("b3", C.c_float), ("nu_scale", C.c_float),
    ]


class TrainParams(C.Structure):
    _fields_ = [
        ("steps", C.c_int32), ("batch", C.c_int32),
        ("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
        ("seed", C.c_uint64),
    ]


def make_params(p: dict) -> Params:
    """SolverParams dict (reference field names, types.ts:3-29) -> wt_params with the reference's
    defaults for the optional fields (tauWall 0.5, interp true, spongeIn 0, f32, regularized)."""
    P = Params()
    P.u = float(p["u"])
    P.nu = float(p["nu"])
    P.cs = float(p.get("cs", 0.0))
    P.sponge_nu = float(p.get("spongeNu", 0.0))
    P.sponge_start = float(p.get("spongeStart", 1.0))
    P.sponge_in = float(p.get("spongeIn", 0.0) or 0.0)
    P.tau_wall = float(p["tauWall"]) if p.get("tauWall") is not None else 0.5
    P.ema_alpha = float(p.get("emaAlpha", 0.0))
    P.init_noise = float(p.get("initNoise", 1e-4))
    P.ground = GROUND[p.get("ground", "freeslip")]
    P.sides = SIDES[p.get("sides", "freeslip")]
    P.precision = PRECISION[p.get("precision", "f32") or "f32"]
    P.interp = 0 if p.get("interp") is False else 1
    P.collision = COLLISION[p.get("collision", "regularized") or "regularized"]
    P.init_mode = INIT[p.get("init", "freestream")]
    P.init_seed = int(p.get("initSeed", 1)) & 0xFFFFFFFF
    return P


def make_wheels(wheels):
    """List of WheelDef dicts {c, axis, r, hw} -> (array, count)."""
    n = len(wheels)
    arr = (Wheel * max(n, 1))()
    for k, w in enumerate(wheels):
        arr[k].c[:] = [float(v) for v in w["c"]]
        arr[k].axis[:] = [float(v) for v in w["axis"]]
        arr[k].r = float(w["r"])
        arr[k].hw = float(w["hw"])
    return arr, n


PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libwt.so")

_lib = None


def _sig(lib):
    P = C.POINTER
    v = C.c_void_p
    i32, i64 = C.c_int32, C.c_int64
    S = C.c_void_p  # wt_solver*
    sigs = {
        "wt_version": ([], C.c_int),
        "wt_error_string": ([C.c_int], C.c_char_p),
        "wt_fits": ([P(Dims), i32, P(i64), P(i32)], C.c_int),
        "wt_pack_params": ([P(Dims), P(Params), P(KParams)], C.c_int),
        "wt_create": ([P(Dims), P(Params), P(S)], C.c_int),
        "wt_destroy": ([S], None),
        "wt_last_error": ([S], C.c_char_p),
        "wt_set_params": ([S, P(Params)], C.c_int),
        "wt_get_params": ([S, P(Params)], C.c_int),
        "wt_get_kparams": ([S, P(KParams)], C.c_int),
        "wt_reset": ([S], C.c_int),
        "wt_clear_stats": ([S], C.c_int),
        "wt_step_count": ([S], i64),
        "wt_upload_flags": ([S, v, i64], C.c_int),
        "wt_upload_sdf": ([S, v, i64], C.c_int),
        "wt_upload_flags_async": ([S, v, i64], C.c_int),
        "wt_upload_sdf_async": ([S, v, i64], C.c_int),
        "wt_set_wheels": ([S, P(Wheel), i32], C.c_int),
        "wt_voxelize": ([S, v, i64, v, i64, v, P(Wheel), i32, P(VoxelInfo)], C.c_int),
        "wt_step": ([S, i32], C.c_int),
        "wt_sample": ([S, P(Stats)], C.c_int),
        "wt_step_and_sample": ([S, i32, P(Stats)], C.c_int),
        "wt_step_and_sample_async": ([S, i32], C.c_int),
        "wt_sample_wait": ([S, P(Stats)], C.c_int),
        "wt_sync": ([S], C.c_int),
        "wt_read_flags": ([S, v, i64], C.c_int),
        "wt_read_sdf": ([S, v, i64], C.c_int),
        "wt_population_bytes": ([S], i64),
        "wt_read_populations": ([S, v, i64], C.c_int),
        "wt_write_populations": ([S, v, i64], C.c_int),
        "wt_read_velocity": ([S, v, i64], C.c_int),
        "wt_read_velocity_half4": ([S, v, i64], C.c_int),
        "wt_read_velocity_half4_async": ([S, v, i64], C.c_int),
        "wt_read_means": ([S, v, v, i64], C.c_int),
        "wt_advect_tracers": ([S, P(TracerParams)], C.c_int),
        "wt_read_tracers": ([S, v, i64, v, i64], C.c_int),
        "wt_write_tracers": ([S, v, i64, v, i64, C.c_uint32], C.c_int),
        "wt_derive_fields": ([S], C.c_int),
        "wt_read_derived": ([S, v, v, v, i64], C.c_int),
        "wt_export_fields": ([S, i32, v, v, v, i64], C.c_int),
        "wt_streamlines": ([S, P(StreamlineParams), v, i64], C.c_int),
        "wt_probes": ([S, v, i32, v], C.c_int),
        "wt_batch_create": ([P(S), i32, P(S)], C.c_int),
        "wt_batch_destroy": ([S], None),
        "wt_batch_last_error": ([S], C.c_char_p),
        "wt_batch_size": ([S], i32),
        "wt_batch_step": ([S, i32], C.c_int),
        "wt_batch_sample": ([S, P(Stats)], C.c_int),
        "wt_batch_set_fused": ([S, i32], C.c_int),
        "wt_set_launch": ([S, i32, i32, i32, i32], C.c_int),
        "wt_get_launch": ([S, P(i32)], C.c_int),
        "wt_autotune": ([S, i32, P(i32)], C.c_int),
        "wt_set_wait_limit": ([S, i64], C.c_int),
        "wt_stream": ([S], v),
        "wt_device": ([S], i32),
        "wt_launch_count": ([S], i64),
        "wt_fused_sample_count": ([S], i64),
        "wt_sample_noalloc": ([P(Dims), P(Params), P(Wheel), i32, v, v, v, v, v, v, v, v], C.c_int),
        "wt_set_closure": ([S, P(Closure)], C.c_int),
        "wt_get_closure": ([S, P(Closure), P(i32)], C.c_int),
        "wt_trainer_create": ([i32, i64, P(S)], C.c_int),
        "wt_trainer_destroy": ([S], None),
        "wt_trainer_last_error": ([S], C.c_char_p),
        "wt_trainer_count": ([S], i64),
        "wt_trainer_clear": ([S], C.c_int),
        "wt_trainer_add_samples": ([S, S, S, C.c_double, C.c_uint64, P(i64)], C.c_int),
        "wt_trainer_put_samples": ([S, v, v, i64], C.c_int),
        "wt_trainer_set_projection_radius": ([S, i32], C.c_int),
        "wt_trainer_read_samples": ([S, i64, i64, v, v], C.c_int),
        "wt_trainer_stats": ([S, v, v], C.c_int),
        "wt_trainer_set_model": ([S, P(Closure)], C.c_int),
        "wt_trainer_get_model": ([S, P(Closure)], C.c_int),
        "wt_trainer_fit": ([S, P(TrainParams), v], C.c_int),
        "wt_trainer_grad": ([S, i64, i64, P(Closure), P(C.c_double)], C.c_int),
        "wt_trainer_infer": ([S, v, i64, v], C.c_int),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


def load(path: str = None):
    """Load libwt.so (built in-tree by windtunnel_vis_b200.build). Raises if it is missing: the
    solver has no CPU fallback."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"libwt.so not found at {p}; build it with `python -m windtunnel_vis_b200.build` "
            "(the CUDA path has no CPU fallback)"
        )
    lib = _sig(C.CDLL(p))
    if path is None:
        _lib = lib
    return lib
