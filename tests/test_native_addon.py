"""The N-API addon (native/wt_napi.c, native/wt_addon.c) and its TypeScript adapter
(native/cuda.ts), which implement the reference's solver interface (src/backend/types.ts:7-53)
on libwt.so.

No JavaScript runtime exists here, so the addon is checked in two ways: wt_napi.c compiles against
the Node-API declarations (tests/napi_stub/node_api.h) and the C ABI header, which catches any
drift between the addon and include/wt.h; and tests/napi_sequence.c, a C program linked to libwt.so
through the addon's own C half, runs the addon's call sequence (create -> uploadFlags -> uploadSdf
-> stepAndSample -> readVelocity -> destroy), whose results must equal the ctypes path's bit for bit.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from windtunnel_vis_b200 import abi, validation as V

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NATIVE = os.path.join(ROOT, "native")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.dirname(abi.LIB_PATH)


def test_addon_compiles_against_the_abi():
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                    "-I", os.path.join(ROOT, "tests", "napi_stub"), "-I", INCLUDE, "-I", NATIVE,
                    os.path.join(NATIVE, "wt_napi.c")], check=True)


@pytest.fixture(scope="module")
def sequence(wtlib, tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("napi") / "napi_sequence")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-O1", "-I", INCLUDE, "-I", NATIVE,
                    os.path.join(ROOT, "tests", "napi_sequence.c"), os.path.join(NATIVE, "wt_addon.c"),
                    "-L", LIBDIR, "-lwt", "-lm", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def _args(params):
    out = []
    for k, v in params.items():
        if isinstance(v, bool):
            v = "true" if v else "false"
        out.append(f"{k}={v}")
    return out


PARAMS = [
    dict(u=0.05, nu=0.004, cs=0.1, ground="freeslip", sides="freeslip", spongeNu=0.03, spongeStart=0.85,
         emaAlpha=0.0, precision="f16"),
    dict(u=0.06, nu=0.0192, cs=0.14, ground="noslip", sides="periodic", spongeNu=0.04, spongeStart=0.84,
         emaAlpha=0.02, tauWall=0.53, spongeIn=0.03, interp=False, collision="bgk"),
    dict(u=0.06, nu=1e-5, cs=0.14, ground="moving", spongeNu=0.03, spongeStart=0.85, emaAlpha=0.0),
]


@pytest.mark.parametrize("params", PARAMS)
def test_addon_maps_solver_params_like_the_python_host(sequence, params):
    out = json.loads(subprocess.run([sequence, "params", *_args(params)], check=True, capture_output=True,
                                    text=True).stdout)
    ref = abi.make_params(dict(params, init="freestream"))
    for k in ("u", "nu", "cs", "sponge_nu", "sponge_start", "sponge_in", "tau_wall", "ema_alpha", "ground", "sides",
              "precision", "interp", "collision", "init_mode"):
        assert out[k] == getattr(ref, k), k


def test_addon_rejects_unknown_enum_strings(sequence):
    out = json.loads(subprocess.run([sequence, "params", "u=0.05", "nu=0.01", "precision=f8"], check=True,
                                    capture_output=True, text=True).stdout)
    assert out == {"error": "precision"}


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f16", "f32"])
def test_addon_call_sequence_matches_ctypes_path(gpu, sequence, tmp_path, prec):
    from windtunnel_vis_b200.solver import Solver

    dims = (96, 48, 48)
    params = dict(PARAMS[0], precision=prec)
    flags, _, sdf = V.round_flags(dims, (28.0, 24.37, 24.21), 5.0, False)
    flags.astype(np.uint32).tofile(tmp_path / "flags.u32")
    sdf.astype(np.float32).tofile(tmp_path / "sdf.f32")
    steps, chunks = 50, 3
    r = subprocess.run([sequence, "run", str(tmp_path), *map(str, dims), str(steps), str(chunks), *_args(params)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    stats = np.fromfile(tmp_path / "stats.f64", np.float64).reshape(chunks, 8)
    vel = np.fromfile(tmp_path / "velocity.f32", np.float32).reshape(-1, 4)
    # the same calls through ctypes (windtunnel_vis_b200.solver), the reference's defaults as the
    # addon applies them (free-stream initial state)
    s = Solver(dims, dict(params, init="freestream"))
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    for c in range(chunks):
        st = s.step_and_sample(steps)
        want = [st["fx"], st["fy"], st["fz"], st["maxU"], st["rhoRef"], float(st["unstable"]), float(st["step"]),
                st["mass"]]
        assert stats[c].tolist() == want, (c, stats[c], want)
    np.testing.assert_array_equal(vel, s.read_velocity())
    s.destroy()
