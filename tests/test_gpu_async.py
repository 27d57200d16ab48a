"""The queued calls (wt_upload_flags_async / wt_upload_sdf_async, wt_step_and_sample_async +
wt_sample_wait, wt_read_velocity_half4_async, wt_sync) give the same bits as the synchronous calls
they mirror, in the same order of geometry changes, steps and samples: statistics, velocity field
and populations. The copies run on the handle's copy streams, so these tests also cover their
ordering: an upload queued while a chunk is in flight applies to the next chunk only, and a
readback queued after a sample holds that sample's field even when the next chunk rewrites it."""
import numpy as np
import pytest
import torch

from windtunnel_vis_b200.solver import Solver, WtError

from .scenes import PARAM_SETS, scene

pytestmark = pytest.mark.gpu


def _pinned(a):
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


def _handles(dims, params, wheels):
    out = []
    for _ in range(2):
        s = Solver(dims, params)
        s.set_wheels(wheels)
        out.append(s)
    return out


def _same_stats(a, b):
    assert a["raw"].tolist() == b["raw"].tolist()
    assert a["mass"] == b["mass"] and a["fluidCells"] == b["fluidCells"] and a["step"] == b["step"]


@pytest.mark.parametrize("prec", ["f16", "f32"])
@pytest.mark.parametrize("dims", [(48, 24, 20), (64, 32, 1)])
def test_queued_pipeline_matches_synchronous_calls(gpu, dims, prec):
    flags, sdf, wheels = scene(dims)
    # a second geometry: the body shifted by one cell along x (flags and distances change)
    flags2 = np.roll(flags.reshape(dims[::-1]), 1, axis=2).ravel()
    sdf2 = np.roll(sdf.reshape(dims[::-1]), 1, axis=2).ravel()
    geoms = [(flags, sdf), (flags, sdf), (flags2, sdf2), (flags2, sdf2)]
    pinned = [(_pinned(f), _pinned(d)) for f, d in geoms]
    n = int(np.prod(dims))
    vel_t = [torch.empty((n, 4), dtype=torch.float16).pin_memory() for _ in geoms]
    a, b = _handles(dims, dict(PARAM_SETS["belt_periodic_les"], precision=prec), wheels)

    # synchronous: upload, stepAndSample, read, one chunk after another
    ref_stats, ref_vel = [], []
    for f, d in geoms:
        a.upload_flags(f)
        a.upload_sdf(d)
        ref_stats.append(a.step_and_sample(12))
        ref_vel.append(a.read_velocity_half())

    # queued: the next chunk's geometry is uploaded while this chunk runs, and this chunk's field
    # is read back while the next one runs
    (f0, _), (d0, _) = pinned[0]
    b.upload_flags_async(f0.numpy())
    b.upload_sdf_async(d0.numpy())
    b.step_and_sample_async(12)
    got = []
    for k in range(len(geoms)):
        if k + 1 < len(geoms):
            (_, fn), (_, dn) = pinned[k + 1]
            b.upload_flags_async(fn)
            b.upload_sdf_async(dn)
        got.append(b.sample_wait())
        b.read_velocity_half_async(vel_t[k].numpy())
        if k + 1 < len(geoms):
            b.step_and_sample_async(12)
    b.sync()
    for k in range(len(geoms)):
        _same_stats(got[k], ref_stats[k])
        np.testing.assert_array_equal(vel_t[k].numpy(), ref_vel[k])
    np.testing.assert_array_equal(b.read_populations(), a.read_populations())
    np.testing.assert_array_equal(b.read_flags(), a.read_flags())
    np.testing.assert_array_equal(b.read_sdf_encoded(), a.read_sdf_encoded())
    a.destroy()
    b.destroy()


def test_readback_keeps_its_sample_while_the_next_chunk_runs(gpu):
    dims = (48, 24, 20)
    flags, sdf, wheels = scene(dims)
    a, b = _handles(dims, dict(PARAM_SETS["freeslip_reg"], precision="f16"), wheels)
    for s in (a, b):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
    a.step_and_sample(30)
    first = a.read_velocity_half()
    a.step_and_sample(30)
    second = a.read_velocity_half()
    assert not np.array_equal(first, second)
    out = torch.empty((a.n, 4), dtype=torch.float16).pin_memory()
    b.step_and_sample(30)
    b.read_velocity_half_async(out.numpy())
    b.step_and_sample_async(30)  # rewrites the field only after the queued copy
    b.sample_wait()
    b.sync()
    np.testing.assert_array_equal(out.numpy(), first)
    np.testing.assert_array_equal(b.read_velocity_half(), second)
    a.destroy()
    b.destroy()


def test_queued_upload_applies_to_every_later_call(gpu):
    dims = (40, 16, 12)
    flags, sdf, wheels = scene(dims)
    s = Solver(dims, dict(PARAM_SETS["freeslip_reg"], precision="f32"))
    s.upload_flags(np.zeros_like(flags))
    s.upload_flags_async(flags)
    np.testing.assert_array_equal(s.read_flags(), flags)  # applied before the read
    s.upload_sdf_async(sdf)
    s.upload_flags_async(np.zeros_like(flags))
    s.upload_flags(flags)  # the synchronous upload comes later and wins
    np.testing.assert_array_equal(s.read_flags(), flags)
    s.destroy()


def test_sample_state_errors(gpu):
    dims = (32, 12, 10)
    flags, sdf, wheels = scene(dims)
    s = Solver(dims, dict(PARAM_SETS["freeslip_reg"], precision="f32"))
    s.upload_flags(flags)
    s.upload_sdf(sdf)
    with pytest.raises(WtError):
        s.sample_wait()  # nothing pending
    s.step_and_sample_async(4)
    for call in (lambda: s.step_and_sample_async(4), lambda: s.sample(), lambda: s.step_and_sample(4)):
        with pytest.raises(WtError):
            call()
    s.step(2)  # plain steps queue behind the pending sample
    st = s.sample_wait()
    assert st["step"] == 4
    assert s.step_and_sample(2)["step"] == 8
    s.destroy()


def test_queued_uploads_apply_to_batch_members(gpu):
    """A queued upload on a batch member applies before the batch's next step, as it does before
    the member's own next step."""
    from windtunnel_vis_b200.solver import Batch

    dims = (40, 16, 12)
    flags, sdf, wheels = scene(dims)
    params = dict(PARAM_SETS["freeslip_reg"], precision="f16")
    alone, member = _handles(dims, params, wheels)
    for s in (alone, member):
        s.upload_flags(np.zeros_like(flags))
        s.step(4)
    alone.upload_flags(flags)
    alone.upload_sdf(sdf)
    member.upload_flags_async(flags)
    member.upload_sdf_async(sdf)
    batch = Batch([member])
    batch.step(6)
    alone.step(6)
    np.testing.assert_array_equal(member.read_populations(), alone.read_populations())
    assert batch.sample()[0]["raw"].tolist() == alone.sample()["raw"].tolist()
    batch.destroy()
    alone.destroy()
    member.destroy()
