"""The tensor-core cache MLP against the FP64 numpy model (oracle/mlp_oracle):
the encoding against its definition, inference (alone and fused with the
composite) and the loss gradient of one batch (same sample selection as
NrcKernel.cu:10-16) against the model with the kernels' own roundings, one
Adam step, and that online training on a known signal drives the loss
down."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as mo
from oracle import oracle as orc
from tests.helpers import INFER_MAX, INFER_MEAN, cache_inference_error, check_cache_gradients
from tfg_b200 import TfgError
from tfg_b200.nrc import BF16, EMA, FP8, FP16, WEIGHTS, ColorMLP, split_layers
from tfg_b200.structs import DATOS_MLP

pytestmark = pytest.mark.gpu

LO, HI = (-6.0, -4.0, -10.0), (6.0, 6.0, 2.0)


def _datos(rng, n, target_fn=None):
    d = np.zeros(n, DATOS_MLP)
    pos = rng.uniform(LO, HI, (n, 3))
    for j, k in enumerate("xyz"):
        d["posicion"][k] = pos[:, j]
        d["direccion"][k] = rng.uniform(0, 1, n)
        d["normal"][k] = rng.uniform(0, 1, n)
    kd = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    for j, k in enumerate("rgb"):
        d["difuso"][k] = kd[:, j]
        d["especular"][k] = 0.0
    y = target_fn(pos, kd) if target_fn else rng.uniform(0, 2, (n, 3))
    for j, k in enumerate("rgb"):
        d["color"][k] = y[:, j]
    return d


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()


def _f16(w):
    return np.asarray(w, np.float32).astype(np.float16).astype(np.float64)


@pytest.fixture(scope="module")
def mlp(built):
    m = ColorMLP(batch=4096, seed=7)
    m.set_bounds(LO, HI)
    yield m
    m.close()


@pytest.mark.parametrize("n", [1000, 128, 5])
def test_inference_matches_fp64_model(mlp, n):
    rng = np.random.default_rng(n)
    d = _datos(rng, n)
    dd = _dev(d)
    out = torch.zeros(n * 3, device="cuda")
    mlp.inference(dd, out, n)
    torch.cuda.synchronize()
    got = out.view(n, 3).cpu().numpy()
    assert np.isfinite(got).all()
    # the GEMM chain: the model with the kernel's roundings on its own operands
    emax, emean = cache_inference_error(mlp, dd, n, got)
    assert emax < INFER_MAX and emean < INFER_MEAN, (emax, emean)
    # the whole pipeline against the FP64 network on the FP64 encoding (before
    # any step inference uses the weights themselves)
    W = [_f16(w) for w in split_layers(mlp.get_params(WEIGHTS))]
    x = mo.encode(mo.rows15(d, LO, HI))
    raw = mo.forward(W, x)[0]
    err = np.abs(got - mo.scrub(raw)) / (np.abs(raw).mean() + 1e-3)
    assert err.max() < 0.02 and err.mean() < 2e-3, (err.max(), err.mean())


# Frequency features: the kernels derive band b from a sine / cosine of
# pi * p by b double-angle steps in FP32, so an error e of the base pair
# grows to about 2^b e; then each feature is rounded to FP16 (half an ulp is
# at most 2^-12 for |x| <= 1).  Inference takes the base pair from the fast
# hardware sine (absolute error about 2^-21.4 on [-pi, pi]), training from
# the accurate sincospif.
BASE_ERR = {"inference": 2.0 ** -20.0, "training": 2.0 ** -23.0}


@pytest.mark.parametrize("which", ["inference", "training"])
def test_encoding_matches_its_definition(mlp, which):
    n = 4000
    d = _datos(np.random.default_rng(77), n)
    x = mlp.encode_features(_dev(d), n, training=which == "training").cpu().numpy().astype(np.float64)
    want = mo.encode(mo.rows15(d, LO, HI))
    bands = np.tile(np.repeat(np.arange(12), 2), 3)
    bound = 2.0 ** -12 + 2.0 ** bands * BASE_ERR[which] * 4.0
    err = np.abs(x[:, :72] - want[:, :72])
    assert (err <= bound[None, :]).all(), f"band error {float((err - bound).max()):.3e} over the bound"
    # the other inputs are FP16 roundings of themselves; the constant 1 and the padding exact
    np.testing.assert_array_equal(x[:, 72:84], mo.round_f16(want[:, 72:84]))
    assert (x[:, 84] == 1.0).all() and (x[:, 85:] == 0.0).all()


def test_inference_composite(mlp):
    rng = np.random.default_rng(3)
    n = 777
    d = _datos(rng, n)
    thr = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    thr[rng.random(n) < 0.4] = 0.0
    img0 = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    img = torch.from_numpy(img0.reshape(-1).copy()).cuda()
    pred = torch.zeros(n * 3, device="cuda")
    dd = _dev(d)
    mlp.inference(dd, pred, n)
    mlp.inference_composite(dd, torch.from_numpy(thr.reshape(-1).copy()).cuda(), img, n)
    torch.cuda.synchronize()
    p = pred.view(n, 3).cpu().numpy()
    want = img0.copy()
    on = (thr > 0).any(axis=1)
    want[on] = img0[on] + thr[on] * p[on]
    np.testing.assert_allclose(img.view(n, 3).cpu().numpy(), want, rtol=1e-6, atol=1e-6)


def _selected(d, n_avail, batch, seed):
    """The samples a training step draws (NrcKernel.cu:10-16) and their targets."""
    idx = np.zeros(batch, np.int32)
    orc.cpu.orc_indices(orc.p(idx), n_avail, batch, seed)
    sel = d[idx]
    return sel, np.stack([sel["color"][k] for k in "rgb"], 1).astype(np.float64)


def test_gradient_matches_fp64_model(mlp):
    rng = np.random.default_rng(11)
    n_avail = 20000
    d = _datos(rng, n_avail)
    g, loss = mlp.compute_gradient(_dev(d), n_avail, seed=5)
    sel, y = _selected(d, n_avail, mlp.batch, 5)
    check_cache_gradients(mlp, _dev(sel), y, g, loss, bias_col=84)
    # and against the exact FP64 network on the FP64 encoding, loosely
    ref_loss, ref = mo.loss_and_grad([_f16(a) for a in split_layers(mlp.get_params(WEIGHTS))],
                                     mo.encode(mo.rows15(sel, LO, HI)), y)
    for l, (gg, rr) in enumerate(zip(split_layers(g), ref)):
        assert np.linalg.norm(gg - rr) / (np.linalg.norm(rr) + 1e-30) < 0.05, l


def test_one_adam_step(built):
    """At t = 1 bias-corrected Adam moves every weight with a non-zero
    gradient by exactly lr against the gradient's sign."""
    m = ColorMLP(batch=1024, seed=3)
    m.set_bounds(LO, HI)
    rng = np.random.default_rng(2)
    d = _datos(rng, 5000)
    dd = _dev(d)
    w0 = m.get_params(WEIGHTS)
    g, _ = m.compute_gradient(dd, 5000, seed=0)
    m.set_hyperparams(lr=1e-3, eps=1e-30)
    m.train_step(dd, 5000)
    w1 = m.get_params(WEIGHTS)
    big = np.abs(g) > 1e-6
    np.testing.assert_allclose(np.abs(w1 - w0)[big], 1e-3, rtol=1e-3)
    assert (np.sign(w1 - w0)[big] == -np.sign(g[big])).mean() > 0.999
    # the weight average starts at zero: after one step it holds (1 - 0.99) w1,
    # and inference uses it debiased by 1 - 0.99^1, i.e. exactly w1
    e1 = m.get_params(EMA)
    np.testing.assert_allclose(e1, 0.01 * w1, rtol=1e-5, atol=1e-9)
    d2 = _datos(np.random.default_rng(5), 300)
    out = torch.zeros(300 * 3, device="cuda")
    m.inference(_dev(d2), out, 300)
    torch.cuda.synchronize()
    emax, emean = cache_inference_error(m, _dev(d2), 300, out.view(300, 3).cpu().numpy())
    assert emax < INFER_MAX and emean < INFER_MEAN, (emax, emean)
    m.close()


def test_small_buffer_is_a_no_op(mlp):
    rng = np.random.default_rng(4)
    d = _datos(rng, 99)
    w0 = mlp.get_params(WEIGHTS)
    assert mlp.train_step(_dev(d), 99) == 0.0
    assert np.array_equal(mlp.get_params(WEIGHTS), w0)


def test_online_training_learns_a_signal(built):
    """Radiance-like target: smooth in position, scaled by albedo."""
    m = ColorMLP(batch=4096, seed=9)
    m.set_bounds(LO, HI)
    rng = np.random.default_rng(8)

    def f(pos, kd):
        base = 0.5 + 0.4 * np.sin(0.7 * pos[:, :1]) * np.cos(0.5 * pos[:, 2:3])
        return base * (0.2 + kd)

    n = 50000
    d = _datos(rng, n, f)
    dd = _dev(d)
    test = _datos(np.random.default_rng(99), 4096, f)
    y = np.stack([test["color"][k] for k in "rgb"], 1)

    def held_out_error():
        out = torch.zeros(4096 * 3, device="cuda")
        m.inference(_dev(test), out, 4096)
        torch.cuda.synchronize()
        p = out.view(-1, 3).cpu().numpy()
        return np.mean((p - y) ** 2 / (y ** 2 + 1e-2))

    before = held_out_error()
    losses = [m.train_step(dd, n) for _ in range(300)]
    assert np.isfinite(losses).all()
    first, last = np.mean(losses[:10]), np.mean(losses[-10:])
    assert last < first / 5, (first, last)
    # inference with the EMA weights tracks the signal on held-out samples
    after = held_out_error()
    assert after < 0.2 * before, (before, after)
    m.close()


def _untrained_reference(m, d):
    W = split_layers(m.get_params(WEIGHTS))
    x = mo.encode(mo.rows15(d, LO, HI))
    return [np.asarray(w, np.float64) for w in W], x


def test_bf16_inference_matches_rounded_model(built):
    m = ColorMLP(batch=4096, seed=21)
    m.set_bounds(LO, HI)
    n = 3000
    d = _datos(np.random.default_rng(21), n)
    W, x = _untrained_reference(m, d)
    m.set_precision(BF16)
    out = torch.zeros(n * 3, device="cuda")
    m.inference(_dev(d), out, n)
    torch.cuda.synchronize()
    got = out.view(n, 3).cpu().numpy()
    want = mo.scrub(mo.forward_quantized(W, x, "bf16"))
    scale = np.abs(mo.forward(W, x)[0]).mean() + 1e-3
    err = np.abs(got - want) / scale
    assert np.isfinite(got).all()
    assert err.mean() < 0.01 and err.max() < 0.08, (err.mean(), err.max())
    m.close()


def test_fp8_inference_matches_quantized_model(built):
    m = ColorMLP(batch=4096, seed=22)
    m.set_bounds(LO, HI)
    n = 4096
    d = _datos(np.random.default_rng(22), n)
    dd = _dev(d)
    W, x = _untrained_reference(m, d)
    m.set_precision(FP8)
    out = torch.zeros(n * 3, device="cuda")
    with pytest.raises(TfgError):          # FP8 needs calibrated scales first
        m.inference(dd, out, n)
    m.calibrate(dd, n)
    m.inference(dd, out, n)
    torch.cuda.synchronize()
    got = out.view(n, 3).cpu().numpy()
    want = mo.scrub(mo.forward_quantized(W, x, "fp8", mo.layer_input_amax(W, x)))
    ref = mo.scrub(mo.forward(W, x)[0])
    scale = np.abs(ref).mean() + 1e-3
    err = np.abs(got - want) / scale
    assert np.isfinite(got).all()
    # One E4M3 step is 12.5 % of a value, and the kernel's scales (from FP16
    # activations) and features (hardware sin/cos) differ from the FP64
    # emulation's by ~1e-3, so individual values round to neighbouring codes:
    # compare on average, and require the kernel to be as accurate against
    # the FP64 network as an exact E4M3 pipeline is.
    assert err.mean() < 0.03, err.mean()
    e_kernel = (np.abs(got - ref) / scale).mean()
    e_exact = (np.abs(want - ref) / scale).mean()
    assert e_kernel < 1.3 * e_exact + 0.01, (e_kernel, e_exact)
    assert e_kernel < 0.15
    # a second call uses the scales re-derived from the first call's amax
    m.inference(dd, out, n)
    torch.cuda.synchronize()
    got2 = out.view(n, 3).cpu().numpy()
    assert (np.abs(got2 - ref) / scale).mean() < 0.15
    m.set_precision(FP16)
    m.close()


@pytest.mark.parametrize("hidden", [3, 7])
def test_other_depths_match_fp64_model(built, hidden):
    """3 and 7 hidden layers: parameter layout, inference and the loss
    gradient against the FP64 model of the same depth."""
    m = ColorMLP(batch=2048, seed=30 + hidden, hidden_layers=hidden)
    m.set_bounds(LO, HI)
    assert m.n_params == 6144 + 4096 * (hidden - 1) + 1024
    w = m.get_params(WEIGHTS)
    W = split_layers(w)
    assert len(W) == hidden + 1 and np.count_nonzero(W[-1][3:]) == 0 and np.count_nonzero(W[0][:, 85:]) == 0
    n = 1500
    d = _datos(np.random.default_rng(hidden), n)
    dd = _dev(d)
    out = torch.zeros(n * 3, device="cuda")
    m.inference(dd, out, n)
    torch.cuda.synchronize()
    emax, emean = cache_inference_error(m, dd, n, out.view(n, 3).cpu().numpy())
    assert emax < INFER_MAX and emean < INFER_MEAN, (emax, emean)
    n_avail = 9000
    dt = _datos(np.random.default_rng(40 + hidden), n_avail)
    g, loss = m.compute_gradient(_dev(dt), n_avail, seed=3)
    sel, y = _selected(dt, n_avail, m.batch, 3)
    check_cache_gradients(m, _dev(sel), y, g, loss, bias_col=84)
    # a few steps on a smooth signal lower the loss
    def f(pos, kd):
        return (0.5 + 0.3 * np.sin(0.7 * pos[:, :1])) * (0.2 + kd)
    ds = _datos(np.random.default_rng(7), 20000, f)
    dd = _dev(ds)
    losses = [m.train_step(dd, 20000) for _ in range(60)]
    assert np.isfinite(losses).all() and np.mean(losses[-5:]) < np.mean(losses[:5]) / 2, losses[::10]
    m.close()


def test_unsupported_depth_is_rejected(built):
    with pytest.raises(TfgError):
        ColorMLP(hidden_layers=4)
