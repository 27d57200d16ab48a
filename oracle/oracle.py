"""Python wrapper of the CPU oracle (oracle/wt_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg. The product package never imports this module.

Parity status: pinned to the reference's lattice tables and validation pass bands; no golden
vectors of the reference exist (it is TypeScript/WGSL and cannot run on these machines).
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from windtunnel_vis_b200 import abi  # noqa: E402  (POD struct layouts of include/wt.h)

from . import build as _build  # noqa: E402

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(path)
        P = C.POINTER
        v = C.c_void_p
        L.or_threads.argtypes = [C.c_int]
        L.or_lattice.argtypes = [C.c_int, v, v, v, v, v, v]
        L.or_pack_params.argtypes = [P(abi.Dims), P(abi.Params), P(abi.KParams)]
        L.or_pack_wheels.argtypes = [P(abi.Wheel), C.c_int, v]
        L.or_encode_sdf.argtypes = [v, C.c_int64, v]
        L.or_encode_sdf.restype = None
        L.or_init.argtypes = [P(abi.Dims), P(abi.KParams), C.c_int, v, v, C.c_int, C.c_uint32, C.c_float]
        L.or_stream_collide.argtypes = [P(abi.Dims), P(abi.KParams), C.c_int, v, v, v, v, v, C.c_int, C.c_int]
        L.or_macro.argtypes = [P(abi.Dims), P(abi.KParams), C.c_int, v, v, v, v, C.c_int, v, v, v, v]
        L.or_voxelize_f32.argtypes = [P(abi.Dims), v, v, C.c_int64, v, v, C.c_int, v, v, v, v, v]
        L.or_voxelize_f64.argtypes = [P(abi.Dims), v, C.c_int64, v, C.c_int64, v, v, v, v]
        L.or_tracers.argtypes = [P(abi.Dims), P(abi.TracerParams), v, v, v, v]
        L.or_derive.argtypes = [P(abi.Dims), C.c_float, v, v, v, v, v, v, v]
        L.or_export.argtypes = [P(abi.Dims), C.c_int, v, v, v, v, v, v]
        L.or_streamlines.argtypes = [P(abi.Dims), P(abi.StreamlineParams), C.c_float, v, v, v, v]
        L.or_probes.argtypes = [P(abi.Dims), v, C.c_int, v, v, v]
        L.or_stream_collide_lc.argtypes = [P(abi.Dims), P(abi.KParams), C.c_int, v, v, v, v, v, C.c_int, C.c_int,
                                           P(abi.Closure)]
        L.or_closure_features.argtypes = [v, v, C.c_int64, C.c_float, v]
        L.or_closure_features.restype = None
        L.or_closure_forward.argtypes = [P(abi.Closure), v, C.c_int64, v]
        L.or_closure_forward.restype = None
        L.or_closure_grad.argtypes = [P(abi.Closure), v, v, C.c_int64, v, v]
        L.or_closure_grad.restype = None
        L.or_pcg.argtypes = [C.c_uint32]
        L.or_pcg.restype = C.c_uint32
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def threads(n=0):
    return lib().or_threads(n)


def lattice(dim):
    q = 19 if dim == 3 else 9
    c = np.zeros((q, 3), np.int32)
    w = np.zeros(q, np.float64)
    t = [np.zeros(q, np.int32) for _ in range(4)]
    lib().or_lattice(dim, _p(c), _p(w), *[_p(x) for x in t])
    return {"q": q, "c": c, "w": w, "opp": t[0], "mirrorY": t[1], "mirrorZ": t[2], "mirrorYZ": t[3]}


def dims_of(dims):
    nx, ny, nz = dims
    return abi.Dims(nx, ny, nz)


def pack_params(dims, params: dict) -> abi.KParams:
    k = abi.KParams()
    rc = lib().or_pack_params(C.byref(dims_of(dims)), C.byref(abi.make_params(params)), C.byref(k))
    assert rc == 0
    return k


def pack_wheels(wheels):
    arr, n = abi.make_wheels(wheels)
    out = np.zeros(8 * 16, np.float32)
    m = lib().or_pack_wheels(arr, n, _p(out))
    return out, m


def encode_sdf(d):
    d = np.ascontiguousarray(d, np.float32)
    out = np.zeros(d.shape, np.uint32)
    lib().or_encode_sdf(_p(d), d.size, _p(out))
    return out


POP_DTYPE = {0: np.float32, 1: np.float16, 2: np.float64}


class OracleSolver:
    """CPU restatement of one solver instance: the same state machine as SolverGPU (init on the
    first step after reset, ping-pong buffers, macro pass at each sample)."""

    def __init__(self, dims, params: dict):
        self.dims = tuple(int(v) for v in dims)
        self.params = dict(params)
        self.prec = abi.PRECISION[params.get("precision", "f32") or "f32"]
        nx, ny, nz = self.dims
        self.n = nx * ny * nz
        self.q = 19 if nz > 1 else 9
        dt = POP_DTYPE[self.prec]
        self.a = np.zeros(self.q * self.n, dt)
        self.b = np.zeros(self.q * self.n, dt)
        self.flags = np.zeros(self.n, np.uint32)
        self.sdf = np.zeros(self.n, np.uint32)
        self.wheels8 = np.zeros(8 * 16, np.float32)
        self.nwheels = 0
        self.vel = np.zeros(4 * self.n, np.float32)
        self.meanA = np.zeros(4 * self.n, np.float32)
        self.meanB = np.zeros(self.n, np.float32)
        self.kp = pack_params(self.dims, self.params)
        self.step_count = 0
        self.pending_init = True
        self.clear_stats()

    def set_params(self, p: dict):
        self.params.update(p)
        self.kp = pack_params(self.dims, self.params)

    def clear_stats(self):
        self.meanA[:] = 0
        self.meanA[3::4] = 1
        self.meanB[:] = 0

    def reset(self):
        self.pending_init = True
        self.step_count = 0
        self.clear_stats()

    def upload_flags(self, flags):
        self.flags[:] = np.asarray(flags, np.uint32).ravel()

    def upload_sdf(self, d):
        self.sdf[:] = encode_sdf(np.asarray(d, np.float32).ravel())

    def set_wheels(self, wheels):
        self.wheels8, self.nwheels = pack_wheels(wheels)

    def _init(self):
        mode = abi.INIT[self.params.get("init", "freestream")]
        seed = int(self.params.get("initSeed", 1)) & 0xFFFFFFFF
        amp = float(self.params.get("initNoise", 1e-4))
        for buf in (self.a, self.b):
            lib().or_init(C.byref(dims_of(self.dims)), C.byref(self.kp), self.prec, _p(self.flags), _p(buf), mode, seed, amp)
        self.pending_init = False

    closure = None

    def set_closure(self, closure):
        """abi.Closure (the learned closure in place of Smagorinsky) or None."""
        self.closure = closure

    def step(self, steps):
        if self.pending_init:
            self._init()
        if self.closure is not None:
            rc = lib().or_stream_collide_lc(C.byref(dims_of(self.dims)), C.byref(self.kp), self.prec, _p(self.a),
                                            _p(self.b), _p(self.flags), _p(self.sdf), _p(self.wheels8), self.nwheels,
                                            int(steps), C.byref(self.closure))
            assert rc == 0, rc
        else:
            lib().or_stream_collide(C.byref(dims_of(self.dims)), C.byref(self.kp), self.prec, _p(self.a), _p(self.b),
                                    _p(self.flags), _p(self.sdf), _p(self.wheels8), self.nwheels, int(steps))
        if steps % 2 == 1:
            self.a, self.b = self.b, self.a
        self.step_count += steps

    @property
    def current(self):
        return self.a

    def sample(self):
        if self.pending_init:
            self._init()
        res = np.zeros(10, np.float64)
        lib().or_macro(C.byref(dims_of(self.dims)), C.byref(self.kp), self.prec, _p(self.a), _p(self.flags),
                       _p(self.sdf), _p(self.wheels8), self.nwheels, _p(self.vel), _p(self.meanA), _p(self.meanB),
                       _p(res))
        return decode_stats(res, self.step_count)

    def step_and_sample(self, steps):
        self.step(steps)
        return self.sample()

    def destroy(self):
        self.a = self.b = None


def decode_stats(d, step):
    """SolverGPU.stepAndSample result decode (SolverGPU.ts:302-308)."""
    return {
        "fx": float(d[0]), "fy": float(d[1]), "fz": float(d[2]),
        "maxU": float(np.sqrt(max(d[3], 0.0))),
        "rhoRef": float(d[4] / d[5]) if d[5] > 0 else 1.0,
        "unstable": bool(d[6] > 0 or not np.isfinite(d[0]) or d[3] > 0.25),
        "step": int(step),
        "raw": np.array(d[:8], np.float64),
        "mass": float(d[8]) if len(d) > 8 else float("nan"),
        "fluidCells": int(d[9]) if len(d) > 9 else -1,
    }


def voxelize_f32(dims, pos, idx, M16, wheels=()):
    nx, ny, nz = dims
    n = nx * ny * nz
    pos = np.ascontiguousarray(pos, np.float32).ravel()
    idx = np.ascontiguousarray(idx, np.uint32).ravel()
    M = np.ascontiguousarray(M16, np.float32).ravel()
    w8, nw = pack_wheels(list(wheels))
    flags = np.zeros(n, np.uint32)
    sdf = np.zeros(n, np.uint32)
    hits = np.zeros(3 * n, np.int32)
    vote = np.zeros(n, np.uint32)
    info = np.zeros(8, np.uint32)
    lib().or_voxelize_f32(C.byref(dims_of(dims)), _p(pos), _p(idx), idx.size // 3, _p(M), _p(w8), nw, _p(flags),
                          _p(sdf), _p(hits), _p(vote), _p(info))
    ok = info[1] > 0
    vinfo = {
        "frontal": int(info[0]), "solidCells": int(info[1]),
        "min": [int(v) for v in info[2:5]] if ok else [0, 0, 0],
        "max": [int(v) + 1 for v in info[5:8]] if ok else [0, 0, 0],
    }
    return flags, sdf, vinfo


def voxelize_f64(dims, pos, idx, M16):
    nx, ny, nz = dims
    n = nx * ny * nz
    pos = np.ascontiguousarray(pos, np.float32).ravel()
    idx = np.ascontiguousarray(idx, np.uint32).ravel()
    M = np.ascontiguousarray(M16, np.float64).ravel()
    flags = np.zeros(n, np.uint8)
    sdf = np.zeros(n, np.float32)
    info = np.zeros(8, np.int32)
    lib().or_voxelize_f64(C.byref(dims_of(dims)), _p(pos), pos.size // 3, _p(idx), idx.size // 3, _p(M), _p(flags),
                          _p(sdf), _p(info))
    return flags, sdf, {"frontal": int(info[0]), "solidCells": int(info[1]), "min": info[2:5].tolist(),
                        "max": info[5:8].tolist()}


def tracers(dims, tp: abi.TracerParams, vel_half4, flags, state, hist):
    """One particle dispatch; state/hist updated in place (float32 arrays)."""
    vel = np.ascontiguousarray(vel_half4, np.float16).view(np.uint16)
    lib().or_tracers(C.byref(dims_of(dims)), C.byref(tp), _p(vel), _p(np.ascontiguousarray(flags, np.uint32)),
                     _p(state), _p(hist))


def pcg(v):
    return lib().or_pcg(v & 0xFFFFFFFF)


def derive(dims, u_ref, vel_half4, flags, meanA, meanB):
    """Derived fields: returns (vort, stat, mean) as float16 arrays of shape (n, 4)."""
    n = dims[0] * dims[1] * dims[2]
    vel = np.ascontiguousarray(vel_half4, np.float16).reshape(n, 4).view(np.uint16)
    outs = [np.zeros((n, 4), np.uint16) for _ in range(3)]
    lib().or_derive(C.byref(dims_of(dims)), float(np.float32(u_ref)), _p(vel), _p(np.ascontiguousarray(flags, np.uint32)),
                    _p(np.ascontiguousarray(meanA, np.float32)), _p(np.ascontiguousarray(meanB, np.float32)),
                    *(_p(o) for o in outs))
    return tuple(o.view(np.float16) for o in outs)


def export(dims, stride, vel_half4, mean_half4, vort_half4):
    """Strided export of half4 fields: {dims, stride, vel, mean, vort} (float32, (points, 4))."""
    o = [-(-d // stride) for d in dims]
    n = o[0] * o[1] * o[2]
    src = [np.ascontiguousarray(a, np.float16).view(np.uint16) for a in (vel_half4, mean_half4, vort_half4)]
    out = [np.zeros((n, 4), np.float32) for _ in range(3)]
    lib().or_export(C.byref(dims_of(dims)), int(stride), *(_p(a) for a in src), *(_p(a) for a in out))
    return {"dims": tuple(o), "stride": stride, "vel": out[0], "mean": out[1], "vort": out[2]}


def streamlines(dims, sp, u_lat, vel_half4, mean_half4, flags):
    """Streamline pass: (seeds * points, 4) float32, seed-major."""
    n = sp.seeds * sp.points
    out = np.zeros((n, 4), np.float32)
    vel = np.ascontiguousarray(vel_half4, np.float16).view(np.uint16)
    mean = np.ascontiguousarray(mean_half4, np.float16).view(np.uint16)
    lib().or_streamlines(C.byref(dims_of(dims)), C.byref(sp), float(np.float32(u_lat)), _p(vel), _p(mean),
                         _p(np.ascontiguousarray(flags, np.uint32)), _p(out))
    return out


def probes(dims, pos4, vel_half4, mean_half4):
    """Probe pass: (count, 8) float32 = instantaneous (ux, uy, uz, rho) and mean."""
    pos = np.ascontiguousarray(pos4, np.float32).reshape(-1, 4)
    out = np.zeros((pos.shape[0], 8), np.float32)
    vel = np.ascontiguousarray(vel_half4, np.float16).view(np.uint16)
    mean = np.ascontiguousarray(mean_half4, np.float16).view(np.uint16)
    lib().or_probes(C.byref(dims_of(dims)), _p(pos), pos.shape[0], _p(vel), _p(mean), _p(out))
    return out


def closure_features(moments, wall, tau0):
    """moments (n x 10: pi xx, yy, zz, xy, xz, yz, rho, ux, uy, uz), wall distances (n) -> the 10
    closure features per row (include/wt.h, wt_closure)."""
    m = np.ascontiguousarray(moments, np.float32).reshape(-1, 10)
    w = np.ascontiguousarray(wall, np.float32).ravel()
    out = np.zeros((m.shape[0], 10), np.float32)
    lib().or_closure_features(_p(m), _p(w), m.shape[0], float(tau0), _p(out))
    return out


def closure_forward(closure, x):
    """nu_t of feature rows x (n x 10) under the network `closure` (abi.Closure)."""
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 10)
    nu = np.zeros(x.shape[0], np.float32)
    lib().or_closure_forward(C.byref(closure), _p(x), x.shape[0], _p(nu))
    return nu


def closure_grad(closure, x, y):
    """(loss, gradient of the 1441 trainable values w1, b1, w2, b2, w3, b3 in field order)."""
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 10)
    y = np.ascontiguousarray(y, np.float32).ravel()
    g = np.zeros(1441, np.float64)
    loss = C.c_double()
    lib().or_closure_grad(C.byref(closure), _p(x), _p(y), x.shape[0], _p(g), C.byref(loss))
    return loss.value, g
