"""Learned closure on the CPU: the oracle's network, gradient and features against an independent
numpy restatement (f64 backpropagation checked by finite differences), the oracle's collision with
a constant closure against the plain method at the raised viscosity, and the host-side helpers."""
import math

import numpy as np
import pytest

from windtunnel_vis_b200 import abi
from windtunnel_vis_b200 import closure as CL

A_GELU = 0.7978845608028654


def bf16(a):
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(A_GELU * (x + 0.044715 * x ** 3)))


def gelu_d(x):
    t = np.tanh(A_GELU * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * A_GELU * (1.0 + 3 * 0.044715 * x * x)


def softplus(z):
    return np.where(z > 20, z, np.log1p(np.exp(np.minimum(z, 20))))


def np_forward(m, x, rounding=True):
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    xn = r((x - m["shift"]) * m["scale"]).astype(np.float64)
    w1, w2, w3 = (r(m[k]).astype(np.float64) for k in ("w1", "w2", "w3"))
    z1 = xn @ w1 + m["b1"]
    h1 = r(gelu(z1)).astype(np.float64)
    z2 = h1 @ w2 + m["b2"]
    h2 = gelu(z2)  # h2 feeds only the CUDA-core output layer: kept in f32 (no bf16 rounding)
    z3 = h2 @ w3 + float(m["b3"])
    return float(m["nu_scale"]) * softplus(z3), (xn, z1, h1, z2, h2, z3, w2, w3)


def np_grad(m, x, y, rounding=True):
    nu, (xn, z1, h1, z2, h2, z3, w2, w3) = np_forward(m, x, rounding)
    ns = float(m["nu_scale"])
    d = (nu - y) / ns
    loss = float(np.mean(d * d))
    dz3 = 2 * d / (1 + np.exp(-z3))
    dz2 = dz3[:, None] * w3[None, :] * gelu_d(z2)
    dz1 = (dz2 @ w2.T) * gelu_d(z1)
    n = x.shape[0]
    g = np.concatenate([(xn.T @ dz1).ravel(), dz1.sum(0), (h1.T @ dz2).ravel(), dz2.sum(0), h2.T @ dz3,
                        [dz3.sum()]]) / n
    return loss, g


def random_case(n, seed=3):
    rng = np.random.default_rng(seed)
    mean = np.array([0, 0, 0, 0, 0, 0, 2e-3, 2.0, 1.0, 0.05])
    std = np.array([1e-4, 1e-4, 1e-4, 5e-5, 5e-5, 5e-5, 1e-3, 0.8, 1e-3, 0.01])
    x = (mean + std * rng.standard_normal((n, 10))).astype(np.float32)
    x[:, 6] = np.abs(x[:, 6])
    x[:, 7] = np.clip(x[:, 7], 0.0, 3.0)
    y = (0.01 * x[:, 6] * (1.0 + np.tanh(x[:, 7] - 1.0))).astype(np.float32)
    m = CL.init_model(seed=seed, shift=mean, scale=1.0 / std, nu_scale=float(np.mean(y)))
    return m, x, y


GROUPS = [("w1", 0, 320), ("b1", 320, 352), ("w2", 352, 1376), ("b2", 1376, 1408), ("w3", 1408, 1440), ("b3", 1440, 1441)]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_numpy_backprop_matches_finite_differences():
    m, x, y = random_case(64)
    for k in ("w1", "w2", "w3", "b1", "b2"):
        m[k] = np.asarray(m[k], np.float64)
    m["b1"] = m["b1"] + 0.1
    _, g = np_grad(m, x.astype(np.float64), y, rounding=False)
    flat = np.concatenate([m["w1"].ravel(), m["b1"], m["w2"].ravel(), m["b2"], m["w3"], [m["b3"]]]).astype(np.float64)
    rng = np.random.default_rng(0)

    def loss_at(v):
        mm = dict(m)
        mm["w1"] = v[0:320].reshape(10, 32)
        mm["b1"] = v[320:352]
        mm["w2"] = v[352:1376].reshape(32, 32)
        mm["b2"] = v[1376:1408]
        mm["w3"] = v[1408:1440]
        mm["b3"] = v[1440]
        return np_grad(mm, x.astype(np.float64), y, rounding=False)[0]

    for p in list(rng.choice(1441, 24, replace=False)) + [1440, 1408, 330]:
        h = 1e-6 * max(1.0, abs(flat[p]))
        vp, vm = flat.copy(), flat.copy()
        vp[p] += h
        vm[p] -= h
        fd = (loss_at(vp) - loss_at(vm)) / (2 * h)
        assert abs(fd - g[p]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(g).max()), (p, fd, g[p])


def test_oracle_gradient_matches_numpy_restatement(oracle):
    m, x, y = random_case(2000)
    loss_o, g_o = oracle.closure_grad(CL.to_struct(m), x, y)
    loss_n, g_n = np_grad(m, x.astype(np.float64), y)
    assert abs(loss_o - loss_n) <= 1e-4 * abs(loss_n)
    for name, a, b in GROUPS:
        # the oracle rounds dz2 and dz1 to bf16 as the training kernel does; numpy keeps them exact
        assert rel(g_o[a:b], g_n[a:b]) < 2e-2, name


def test_oracle_forward_matches_numpy_restatement(oracle):
    m, x, y = random_case(3000, seed=5)
    nu_o = oracle.closure_forward(CL.to_struct(m), x)
    nu_n, _ = np_forward(m, x.astype(np.float64))
    # identical rounding points; the f32 accumulation order and bf16 ties are the only differences
    assert np.max(np.abs(nu_o - nu_n) / (np.abs(nu_n) + 1e-3 * float(m["nu_scale"]))) < 2e-2
    assert np.median(np.abs(nu_o - nu_n) / np.abs(nu_n)) < 1e-5


def test_oracle_features_match_definition(oracle):
    rng = np.random.default_rng(7)
    n = 500
    mo = np.zeros((n, 10), np.float32)
    mo[:, :6] = 1e-4 * rng.standard_normal((n, 6))
    mo[:, 6] = 1.0 + 1e-3 * rng.standard_normal(n)
    mo[:, 7:10] = 0.05 * rng.standard_normal((n, 3))
    wall = rng.uniform(0, 3, n).astype(np.float32)
    tau0 = 0.503
    x = oracle.closure_features(mo, wall, tau0)
    p = mo[:, :6].astype(np.float64)
    pn = np.sqrt(p[:, 0] ** 2 + p[:, 1] ** 2 + p[:, 2] ** 2 + 2 * (p[:, 3] ** 2 + p[:, 4] ** 2 + p[:, 5] ** 2))
    rho = mo[:, 6].astype(np.float64)
    ts = 0.5 * (tau0 + np.sqrt(tau0 ** 2 + 18 * math.sqrt(2) * 0.01 * pn / rho))
    S = 3 * pn / (math.sqrt(2) * rho * ts)
    assert np.allclose(x[:, :6], mo[:, :6])
    assert np.allclose(x[:, 6], S, rtol=1e-5)
    assert np.array_equal(x[:, 7], wall)
    assert np.array_equal(x[:, 8], mo[:, 6])
    assert np.allclose(x[:, 9], np.linalg.norm(mo[:, 7:10].astype(np.float64), axis=1), rtol=1e-6)
    # Smagorinsky's nu_t from the strain feature is (tau_s - tau0) / 3 at Cs = 0.1
    assert np.allclose(CL.smagorinsky_nu(x), (ts - tau0) / 3, rtol=1e-4)


def constant_closure(nu_c, nu_scale=1e-3):
    m = CL.init_model(seed=1, nu_scale=nu_scale)
    m["w1"][:] = 0
    m["w2"][:] = 0
    m["w3"][:] = 0
    m["b3"] = np.float32(math.log(math.expm1(nu_c / nu_scale)))
    return m


def sphere_setup(dims, r, c):
    from windtunnel_vis_b200.validation import round_flags

    flags, frontal, sdf = round_flags(dims, c, r, False)
    return flags, sdf


@pytest.mark.parametrize("collision", ["regularized", "bgk"])
def test_oracle_constant_closure_equals_raised_viscosity(oracle, collision):
    dims = (24, 12, 12)
    flags, sdf = sphere_setup(dims, 2.5, (8.0, 6.2, 6.1))
    nu, nu_c = 0.01, 2e-3
    base = dict(u=0.05, nu=nu, cs=0.0, collision=collision, spongeStart=0.8, spongeNu=0.02)
    a = oracle.OracleSolver(dims, base)
    b = oracle.OracleSolver(dims, dict(base, nu=nu + nu_c))
    for s in (a, b):
        s.upload_flags(flags)
        s.upload_sdf(sdf)
    a.set_closure(CL.to_struct(constant_closure(nu_c)))
    a.step(6)
    b.step(6)
    assert np.max(np.abs(a.current - b.current)) < 2e-6


def test_model_struct_round_trip_and_flat_order():
    m = CL.init_model(seed=4, shift=np.arange(10), scale=np.ones(10) * 2, nu_scale=3e-4)
    back = CL.from_struct(CL.to_struct(m))
    for k in m:
        assert np.array_equal(np.asarray(back[k], np.float32), np.asarray(m[k], np.float32)), k
    flat = CL.flat_params(m)
    assert flat.size == CL.N_PARAM == 1441
    raw = np.frombuffer(bytes(CL.to_struct(m)), np.float32)
    assert np.array_equal(raw[20:20 + 1441], flat)  # w1 .. b3 are contiguous in wt_closure


def test_seeded_bodies_and_fields():
    bodies = CL.seeded_bodies(8, seed=11)
    assert [b["kind"] for b in bodies[:3]] == ["sphere", "box", "ellipsoid"]
    assert all(1.0 <= b["aspect"] <= 4.0 for b in bodies)
    assert bodies == CL.seeded_bodies(8, seed=11)
    for b in bodies[:3]:
        fine, ff, fs = CL.body_fields((128, 64, 64), b)
        coarse, cf, cs = CL.body_fields((64, 32, 32), b)
        vf, vc = int(fine.sum()), int(coarse.sum())
        assert vf > 0 and vc > 0
        assert abs(vf / 8 - vc) / vc < 0.2  # same body at half the resolution
        assert np.all(fs[(fine == 1) & (fs >= 0)] <= 2.5)


def test_a_priori_metrics():
    y = np.linspace(0, 1, 100)
    assert CL.a_priori_metrics(y, y)["nmse"] == 0.0
    assert abs(CL.a_priori_metrics(np.full(100, y.mean()), y)["nmse"] - 1.0) < 1e-12


def test_pretrained_network_is_gated_to_its_regime(tmp_path):
    # the shipped network carries the Reynolds-number range it was trained and checked in
    m = CL.load_pretrained(1000.0)
    lo, hi = (float(v) for v in m["regime_re"])
    assert lo <= 1000.0 <= hi and hi < 3000.0
    CL.to_struct(m)  # the regime entry does not disturb the network's layout
    for re in (lo / 2.0, 3000.0, 1e4, 2e4 * 0.336):
        with pytest.raises(CL.ClosureRegimeError):
            CL.load_pretrained(re)
    assert float(CL.load_pretrained(1e4, allow_outside=True)["b3"]) == float(m["b3"])
    # a network saved with a regime round-trips it; one saved without has none and is never refused
    path = tmp_path / "net.npz"
    CL.save(CL.init_model(seed=3), path, regime={"re": (100.0, 400.0)})
    CL.load_pretrained(200.0, path=str(path))
    with pytest.raises(CL.ClosureRegimeError):
        CL.load_pretrained(800.0, path=str(path))
    CL.save(CL.init_model(seed=3), path)
    CL.load_pretrained(1e6, path=str(path))
