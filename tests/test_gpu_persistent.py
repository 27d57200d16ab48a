"""The persistent kernel: many lattice updates of one tunnel (WT_LAUNCH_PERSISTENT) or of a batch of
tunnels (WT_BATCH_PERSISTENT) in one cooperative launch, the steps separated by a grid-wide
barrier. Every cell goes through the per-step kernels' device code, so the populations and the
statistics are bit-identical to the same steps taken by the per-step kernels, on every boundary path
of the parity scenes."""
import numpy as np
import pytest

from windtunnel_vis_b200 import abi, validation as V
from windtunnel_vis_b200.solver import Batch, Solver

from .scenes import PARAM_SETS, scene

pytestmark = pytest.mark.gpu

PERSISTENT = (abi.WT_LAUNCH_PERSISTENT, 2, 0, 0)


def _solver(dims, params, launch=None):
    flags, sdf, wheels = scene(dims)
    s = Solver(dims, params)
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    s.set_wheels(wheels)
    if launch:
        s.set_launch(*launch)
    return s


@pytest.mark.parametrize("prec", ["f16", "f32"])
@pytest.mark.parametrize("pset", list(PARAM_SETS))
@pytest.mark.parametrize("dims", [(32, 14, 12), (34, 14, 10), (48, 16, 1), (160, 12, 1)])
def test_persistent_steps_match_per_step_kernels(gpu, dims, pset, prec):
    params = dict(PARAM_SETS[pset], precision=prec)
    a = _solver(dims, params)
    b = _solver(dims, params, PERSISTENT)
    assert b.get_launch() == PERSISTENT
    for n in (1, 7, 24):
        a.step(n)
        l0 = b.launches
        b.step(n)
        if n == 24:
            assert b.launches == l0 + 1  # the 24 steps in one launch
        np.testing.assert_array_equal(a.read_populations(), b.read_populations())
    sa, sb = a.step_and_sample(10), b.step_and_sample(10)
    assert sa["raw"].tolist() == sb["raw"].tolist() and sa["mass"] == sb["mass"]
    np.testing.assert_array_equal(a.read_velocity_half(), b.read_velocity_half())
    a.destroy()
    b.destroy()


QUEUE = (abi.WT_LAUNCH_QUEUE, 2, 0, 0)


@pytest.mark.parametrize("prec", ["f16", "f32"])
@pytest.mark.parametrize("pset", list(PARAM_SETS))
@pytest.mark.parametrize("dims", [(32, 14, 12), (34, 14, 10), (48, 16, 1), (160, 12, 1)])
def test_queue_steps_match_per_step_kernels(gpu, dims, pset, prec):
    # one work-queue launch per step (captured in the step graphs; the counter clears itself), the
    # sampling step on the per-step kernels: bit-identical to the per-step kernels throughout
    params = dict(PARAM_SETS[pset], precision=prec)
    a = _solver(dims, params)
    b = _solver(dims, params, QUEUE)
    assert b.get_launch() == QUEUE
    for n in (1, 7, 24, 3):
        a.step(n)
        b.step(n)
        np.testing.assert_array_equal(a.read_populations(), b.read_populations())
        sa, sb = a.step_and_sample(11), b.step_and_sample(11)
        assert sa["raw"].tolist() == sb["raw"].tolist() and sa["mass"] == sb["mass"]
    np.testing.assert_array_equal(a.read_velocity_half(), b.read_velocity_half())
    a.destroy()
    b.destroy()


def test_persistent_channel_matches_graph_steps(gpu):
    # the D2Q9 cylinder channel (512 x 128, FP32, BGK): 500 updates as one launch
    dims = V.CHANNEL_DIMS
    params = V.channel_params("f32")
    flags, _, sdf = V.channel_geometry()
    out = []
    for launch in (None, PERSISTENT):
        s = Solver(dims, params)
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        if launch:
            s.set_launch(*launch)
        st = s.step_and_sample(500)
        out.append((s.read_populations(), st["raw"].tolist()))
        s.destroy()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]


@pytest.mark.parametrize("prec", ["f16", "f32"])
def test_persistent_batch_matches_members_stepped_alone(gpu, prec):
    # tunnels of different sizes and parameters (same lattice, storage and collision) in one launch
    cases = [((32, 14, 12), "belt_periodic_les"), ((48, 16, 14), "freeslip_reg"), ((64, 12, 10), "belt_periodic_les")]
    alone = [_solver(d, dict(PARAM_SETS[p], precision=prec)) for d, p in cases]
    members = [_solver(d, dict(PARAM_SETS[p], precision=prec)) for d, p in cases]
    batch = Batch(members, persistent=True)
    for n in (3, 16, 9):
        for s in alone:
            s.step(n)
        l0 = members[0].launches
        batch.step(n)
        if n == 16:
            assert members[0].launches == l0 + 1  # one launch for every member's 16 steps
        for s, t in zip(alone, members):
            np.testing.assert_array_equal(s.read_populations(), t.read_populations())
    for s, st in zip(alone, batch.sample()):
        assert s.sample()["raw"].tolist() == st["raw"].tolist()
    batch.destroy()
    for s in alone + members:
        s.destroy()


@pytest.mark.parametrize("prec", ["f16", "f32"])
def test_queue_batch_matches_members_stepped_alone(gpu, prec):
    # the work queue launched once per step under the batch graphs (read-only-cache loads, no grid
    # barrier): bit-identical to the members stepped alone, one launch per step for all members
    cases = [((32, 14, 12), "belt_periodic_les"), ((48, 16, 14), "freeslip_reg"), ((64, 12, 10), "belt_periodic_les")]
    alone = [_solver(d, dict(PARAM_SETS[p], precision=prec)) for d, p in cases]
    members = [_solver(d, dict(PARAM_SETS[p], precision=prec)) for d, p in cases]
    batch = Batch(members, queue=True)
    for n in (3, 16, 9, 24):
        for s in alone:
            s.step(n)
        l0 = [t.launches for t in members]
        batch.step(n)
        if n == 16:
            # graph replays: one work-queue launch per step, counted on the first member
            assert members[0].launches == l0[0] + 16 and [t.launches for t in members[1:]] == l0[1:]
        for s, t in zip(alone, members):
            np.testing.assert_array_equal(s.read_populations(), t.read_populations())
    for s, st in zip(alone, batch.sample()):
        assert s.sample()["raw"].tolist() == st["raw"].tolist()
    batch.destroy()
    for s in alone + members:
        s.destroy()
