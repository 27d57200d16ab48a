"""The C ABI: libwt.so loads without a GPU, exports every entry point include/wt.h declares, and
the ctypes mirror (windtunnel_vis_b200/abi.py) matches the header's struct layouts."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from windtunnel_vis_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include"))) if h.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(wt_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_the_surface():
    names = declared_functions()
    for must in ("wt_create", "wt_destroy", "wt_step_and_sample", "wt_upload_flags", "wt_upload_sdf", "wt_voxelize",
                 "wt_advect_tracers", "wt_read_populations", "wt_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(wtlib):
    lib = C.CDLL(abi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.wt_version() == 2


STRUCTS = {
    "wt_dims": abi.Dims, "wt_params": abi.Params, "wt_kparams": abi.KParams, "wt_stats": abi.Stats,
    "wt_wheel": abi.Wheel, "wt_voxel_info": abi.VoxelInfo, "wt_tracer_params": abi.TracerParams,
    "wt_streamline_params": abi.StreamlineParams, "wt_closure": abi.Closure, "wt_train_params": abi.TrainParams,
}


def test_struct_layouts_match_header():
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "wt.h"', "int main(void){"]
    for cname, cls in STRUCTS.items():
        src.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            src.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    src.append("return 0;}")
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "layout.c")
        exe = os.path.join(td, "layout")
        open(c, "w").write("\n".join(src))
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line)
    for cname, cls in STRUCTS.items():
        assert int(got[f"{cname} size"]) == C.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(cls, f).offset, (cname, f)
    assert C.sizeof(abi.KParams) == 96  # the reference's 96-byte Params uniform


def test_pack_params_library_matches_oracle(wtlib, oracle):
    from windtunnel_vis_b200.solver import pack_params

    for dims, p in [((256, 128, 128), dict(u=0.05, nu=0.004, cs=0.1, ground="moving", sides="periodic", spongeNu=0.03,
                                           spongeStart=0.85, spongeIn=0.03, tauWall=0.53, emaAlpha=0.02)),
                    ((512, 128, 1), dict(u=0.05, nu=0.01, cs=0.0, ground="freeslip", collision="bgk", interp=False))]:
        a, b = pack_params(dims, p), oracle.pack_params(dims, p)
        assert bytes(a) == bytes(b)


def test_errors_without_device_are_reported(wtlib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    h = C.c_void_p()
    P = abi.make_params(dict(u=0.05, nu=0.01))
    rc = wtlib.wt_create(C.byref(abi.Dims(8, 8, 8)), C.byref(P), C.byref(h))
    assert rc == abi.WT_E_NO_DEVICE
    assert b"no CUDA device" in wtlib.wt_last_error(None)
    rc = wtlib.wt_create(C.byref(abi.Dims(0, 8, 8)), C.byref(P), C.byref(h))
    assert rc == abi.WT_E_INVALID


def test_sample_noalloc_argument_checks_without_device(wtlib):
    # size and argument checks come before any CUDA call, so they hold on a machine without a GPU
    P = abi.make_params(dict(u=0.05, nu=0.01, precision="f16"))
    dummy = C.c_void_p(4096)  # never dereferenced: every call below is rejected first
    args = [None, 0] + [dummy] * 7 + [None]
    rc = wtlib.wt_sample_noalloc(C.byref(abi.Dims(256, 128, 129)), C.byref(P), *args)
    assert rc == abi.WT_E_INVALID
    assert b"exceed the limit of 4194304 cells" in wtlib.wt_last_error(None)
    rc = wtlib.wt_sample_noalloc(C.byref(abi.Dims(0, 8, 8)), C.byref(P), *args)
    assert rc == abi.WT_E_INVALID
    rc = wtlib.wt_sample_noalloc(C.byref(abi.Dims(8, 8, 8)), C.byref(P), None, 17, *args[2:])
    assert rc == abi.WT_E_INVALID


def test_trainer_without_device_is_reported(wtlib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is visible")
    h = C.c_void_p()
    assert wtlib.wt_trainer_create(0, 16, C.byref(h)) == abi.WT_E_NO_DEVICE
    assert wtlib.wt_trainer_create(0, -1, C.byref(h)) == abi.WT_E_INVALID
