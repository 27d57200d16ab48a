"""wt_sample_noalloc (the sampling pass on caller-owned buffers, reduction scratch in a fixed
device array) against wt_sample on a handle holding the same state.

The caller's buffers come from torch's allocator, the way a host that owns all device memory would
hand them over. Two calls in a row go through the one shared scratch array: a 3-D f16 tunnel, then
a smaller 2-D f32 one, so the second call runs over what the first left in the array. Tolerances
are the parity tests': force sums relative 5e-3 (f16) / 1e-4 (f32), counts exact, EMA means
relative 5e-3 / 1e-4, velocity field absolute 1e-4 / 2e-6.
"""
import ctypes as C

import numpy as np
import pytest

from windtunnel_vis_b200 import abi
from windtunnel_vis_b200.solver import Solver

from .scenes import PARAM_SETS, scene

pytestmark = pytest.mark.gpu

STAT_RTOL = {"f32": 1e-4, "f16": 5e-3}
MEAN_RTOL = {"f32": 1e-4, "f16": 5e-3}
VEL_ATOL = {"f32": 2e-6, "f16": 1e-4}
COUNTS = (5, 6, 7)  # n_ref, nan count, solid count


def _device_copy(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _check_one(torch, lib, dims, params, steps):
    prec = params["precision"]
    flags, sdf, wheels = scene(dims)
    s = Solver(dims, params)
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    s.set_wheels(wheels)
    s.step(steps)

    # the caller's own device buffers, holding the handle's current state
    pops = _device_copy(torch, s.read_populations())
    dflags = _device_copy(torch, s.read_flags().view(np.int32))
    dsdf = _device_copy(torch, s.read_sdf_encoded().view(np.int32))
    m4, mb = s.read_means()
    dm4, dmb = _device_copy(torch, m4), _device_copy(torch, mb)
    vel = torch.full((s.n, 4), float("nan"), dtype=torch.float16, device="cuda")
    result = torch.full((8,), float("nan"), dtype=torch.float64, device="cuda")

    w, nw = abi.make_wheels(wheels)
    stream = torch.cuda.current_stream()
    rc = lib.wt_sample_noalloc(C.byref(abi.Dims(*dims)), C.byref(abi.make_params(params)), w, nw,
                               pops.data_ptr(), dflags.data_ptr(), dsdf.data_ptr(), vel.data_ptr(), dm4.data_ptr(),
                               dmb.data_ptr(), result.data_ptr(), C.c_void_p(stream.cuda_stream))
    assert rc == 0, lib.wt_last_error(None).decode()
    torch.cuda.synchronize()

    ref = s.sample()
    ref_m4, ref_mb = s.read_means()
    ref_vel = s.read_velocity()
    got = result.cpu().numpy()
    raw = ref["raw"]
    for k in (0, 1, 2):
        assert abs(got[k] - raw[k]) <= STAT_RTOL[prec] * max(abs(raw[k]), 1e-6), (k, got[k], raw[k])
    assert got[3] == pytest.approx(raw[3], rel=STAT_RTOL[prec])
    assert got[4] == pytest.approx(raw[4], rel=STAT_RTOL[prec])
    for k in COUNTS:
        assert got[k] == raw[k], (k, got[k], raw[k])
    assert raw[7] > 0 and raw[0] != 0  # the scene has solids and a non-zero drag
    np.testing.assert_allclose(dm4.cpu().numpy(), ref_m4, rtol=MEAN_RTOL[prec], atol=1e-7)
    np.testing.assert_allclose(dmb.cpu().numpy(), ref_mb, rtol=MEAN_RTOL[prec], atol=1e-7)
    np.testing.assert_allclose(vel.float().cpu().numpy(), ref_vel, rtol=0, atol=VEL_ATOL[prec])
    s.destroy()


def test_sample_noalloc_matches_sample_twice(gpu):
    import torch

    lib = gpu
    torch.cuda.init()
    _check_one(torch, lib, (32, 14, 12), dict(PARAM_SETS["belt_periodic_les"], precision="f16"), 25)
    _check_one(torch, lib, (48, 16, 1), dict(PARAM_SETS["freeslip_reg"], precision="f32"), 15)


def test_sample_noalloc_allocates_no_device_memory(gpu):
    # after a first call (which may load the library's device code), further calls leave the
    # device's free memory unchanged
    import torch

    lib = gpu
    dims = (32, 14, 12)
    params = dict(PARAM_SETS["freeslip_reg"], precision="f16")
    flags, sdf, wheels = scene(dims)
    n = dims[0] * dims[1] * dims[2]
    s = Solver(dims, params)
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    s.step(5)
    pops = _device_copy(torch, s.read_populations())
    dflags = _device_copy(torch, s.read_flags().view(np.int32))
    dsdf = _device_copy(torch, s.read_sdf_encoded().view(np.int32))
    m4, mb = s.read_means()
    dm4, dmb = _device_copy(torch, m4), _device_copy(torch, mb)
    vel = torch.zeros((n, 4), dtype=torch.float16, device="cuda")
    result = torch.zeros((8,), dtype=torch.float64, device="cuda")
    s.destroy()
    w, nw = abi.make_wheels(wheels)

    def call():
        rc = lib.wt_sample_noalloc(C.byref(abi.Dims(*dims)), C.byref(abi.make_params(params)), w, nw,
                                   pops.data_ptr(), dflags.data_ptr(), dsdf.data_ptr(), vel.data_ptr(),
                                   dm4.data_ptr(), dmb.data_ptr(), result.data_ptr(), None)
        assert rc == 0, lib.wt_last_error(None).decode()
        torch.cuda.synchronize()

    call()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        call()
    assert torch.cuda.mem_get_info()[0] == free0


def test_sample_noalloc_rejects_grids_above_the_limit(gpu):
    import torch

    lib = gpu
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    dims = abi.Dims(256, 128, 129)  # one plane more than the limit allows
    rc = lib.wt_sample_noalloc(C.byref(dims), C.byref(abi.make_params(dict(u=0.05, nu=0.01, precision="f16"))),
                               None, 0, p, p, p, p, p, p, p, None)
    assert rc == abi.WT_E_INVALID
    assert "exceed the limit of 4194304 cells" in lib.wt_last_error(None).decode()
