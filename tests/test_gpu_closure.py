"""Learned closure on the GPU, through libwt.so, against the CPU oracle.

  tensor-core inference (wt_trainer_infer) vs oracle forward ...... |d nu| <= 2e-2 |nu| + 1e-3 nu_scale
  training gradient (wt_trainer_grad) vs oracle gradient .......... relative L2 <= 3e-2 per tensor
  stream-collide with a network (bulk on tcgen05, face and wall
    cells on CUDA cores) vs oracle with the same network ......... f32 |d f| <= 2e-6 (1 step),
                                                                    1e-5 (10 steps); f16 5e-4
  constant network vs the plain method at nu + nu_c ............... f32 |d f| <= 2e-6
The differences come from tanh.approx.f32 inside gelu (the oracle uses tanh), which can move a
bf16 rounding of a hidden activation by one unit, and from the order of the f32 accumulations.
"""
import math

import numpy as np
import pytest

from windtunnel_vis_b200 import closure as CL
from windtunnel_vis_b200.solver import Solver, WtError

from .scenes import PARAM_SETS, scene
from .test_closure import constant_closure, random_case, rel, GROUPS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trainer(gpu):
    t = CL.Trainer(1 << 16)
    yield t
    t.destroy()


def test_tensor_core_inference_matches_oracle(trainer, oracle):
    m, x, y = random_case(1000, seed=11)  # 1000 rows: the last block is partly padding
    trainer.set_model(m)
    nu_g = trainer.infer(x)
    nu_o = oracle.closure_forward(CL.to_struct(m), x)
    assert np.all(np.isfinite(nu_g))
    err = np.abs(nu_g - nu_o) / (np.abs(nu_o) + 1e-3 * float(m["nu_scale"]))
    assert err.max() < 2e-2, err.max()
    assert np.median(err) < 2e-3


def test_training_gradient_matches_oracle(trainer, oracle):
    m, x, y = random_case(3000, seed=12)
    trainer.clear()
    trainer.put_samples(x, y)
    trainer.set_model(m)
    loss_g, g_g = trainer.grad(0, 3000)
    loss_o, g_o = oracle.closure_grad(CL.to_struct(m), x, y)
    assert abs(loss_g - loss_o) <= 2e-3 * loss_o
    for name, a, b in GROUPS:
        assert rel(g_g[a:b], g_o[a:b]) < 3e-2, (name, rel(g_g[a:b], g_o[a:b]))
    # a sub-range of the pool
    loss_g2, g_g2 = trainer.grad(1000, 700)
    loss_o2, g_o2 = oracle.closure_grad(CL.to_struct(m), x[1000:1700], y[1000:1700])
    assert abs(loss_g2 - loss_o2) <= 2e-3 * loss_o2
    assert rel(g_g2, g_o2) < 3e-2


def test_adam_fit_reduces_the_loss(trainer, oracle):
    m, x, y = random_case(1 << 14, seed=13)
    trainer.clear()
    trainer.put_samples(x, y)
    trainer.set_model(m)
    loss0, _ = trainer.grad(0, 1 << 14)
    hist = trainer.fit(400, batch=4096, lr=3e-3, seed=5)
    assert hist.shape == (400,) and np.all(np.isfinite(hist))
    loss1, _ = trainer.grad(0, 1 << 14)
    assert loss1 < 0.2 * loss0, (loss0, loss1)
    # the trained network, read back, is the one the oracle evaluates
    mt = trainer.get_model()
    nu_g = trainer.infer(x[:2000])
    nu_o = oracle.closure_forward(CL.to_struct(mt), x[:2000])
    assert np.max(np.abs(nu_g - nu_o) / (np.abs(nu_o) + 1e-3 * float(mt["nu_scale"]))) < 2e-2
    # same seed, same model: the fit is deterministic
    trainer.set_model(m)
    hist2 = trainer.fit(400, batch=4096, lr=3e-3, seed=5)
    assert np.array_equal(hist, hist2)


def _scene_pair(oracle, dims, params, model):
    flags, sdf, wheels = scene(dims)
    g = Solver(dims, params)
    o = oracle.OracleSolver(dims, params)
    for s in (g, o):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        s.set_wheels(wheels)
    g.set_closure(model)
    o.set_closure(CL.to_struct(model))
    return g, o


def _scene_model(seed=21, nu_scale=2e-3):
    m, _, _ = random_case(16, seed=seed)
    m["nu_scale"] = np.float32(nu_scale)
    return m


@pytest.mark.parametrize("pset", list(PARAM_SETS))
@pytest.mark.parametrize("dims", [(32, 14, 12), (64, 16, 12), (300, 12, 8)])
def test_stream_collide_with_network_matches_oracle(gpu, oracle, dims, pset):
    params = dict(PARAM_SETS[pset], precision="f32", init="freestream")
    m = _scene_model()
    g, o = _scene_pair(oracle, dims, params, m)
    for steps, tol in ((1, 2e-6), (9, 1e-5)):
        g.step(steps)
        o.step(steps)
        d = np.abs(g.read_populations().astype(np.float64) - o.current.astype(np.float64))
        assert d.max() <= tol, (steps, d.max())
    # the network changed the run: the plain method differs by far more than the tolerance
    p = oracle.OracleSolver(dims, params)
    flags, sdf, wheels = scene(dims)
    p.upload_flags(flags)
    p.upload_sdf(sdf)
    p.set_wheels(wheels)
    p.step(10)
    assert np.abs(p.current.astype(np.float64) - o.current.astype(np.float64)).max() > 10 * 1e-5
    assert g.get_closure() is not None
    g.destroy()


def test_stream_collide_with_network_f16(gpu, oracle):
    dims = (64, 16, 12)
    params = dict(PARAM_SETS["freeslip_reg"], precision="f16", init="freestream")
    g, o = _scene_pair(oracle, dims, params, _scene_model())
    g.step(5)
    o.step(5)
    d = np.abs(g.read_populations().astype(np.float64) - o.current.astype(np.float64))
    assert d.max() <= 5e-4, d.max()
    g.destroy()


@pytest.mark.parametrize("collision", ["regularized", "bgk"])
def test_constant_network_equals_raised_viscosity(gpu, collision):
    dims = (64, 16, 12)
    flags, sdf, wheels = scene(dims)
    nu_c = 3e-3
    base = dict(PARAM_SETS["freeslip_reg"], cs=0.0, collision=collision, precision="f32", init="freestream")
    a = Solver(dims, base)
    b = Solver(dims, dict(base, nu=base["nu"] + nu_c))
    for s in (a, b):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
        s.set_wheels(wheels)
    a.set_closure(constant_closure(nu_c))
    a.step(10)
    b.step(10)
    d = np.abs(a.read_populations().astype(np.float64) - b.read_populations().astype(np.float64))
    assert d.max() <= 2e-6, d.max()
    # removing the network restores the plain method exactly
    a.set_closure(None)
    assert a.get_closure() is None
    a.destroy()
    b.destroy()


def test_closure_rejects_unsupported_handles(gpu):
    m = _scene_model()
    s = Solver((32, 16, 1), dict(u=0.05, nu=0.02))
    with pytest.raises(WtError):
        s.set_closure(m)
    s.destroy()
    s = Solver((32, 8, 8), dict(u=0.05, nu=0.02, precision="f64"))
    with pytest.raises(WtError):
        s.set_closure(m)
    s.destroy()
    s = Solver((33, 8, 8), dict(u=0.05, nu=0.02))
    with pytest.raises(WtError):
        s.set_closure(m)
    s.destroy()
