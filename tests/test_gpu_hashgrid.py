"""The cache model with the reference's own input encoding (hash grid on the
position, one-blob on direction and normal, identity on the albedos) against
the FP64 oracle: inference, the gradients of the layers and of the hash-grid
tables, online training, checkpoints, the other inference precisions and a
whole cache frame."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as mo
from oracle import oracle as orc
from tests.helpers import INFER_MAX, INFER_MEAN, cache_inference_error, check_cache_gradients
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
from tfg_b200.nrc import (BF16, EMA, FP8, HASHGRID, WEIGHTS, ColorMLP, NrcRenderer, hashgrid_reference,
                          one_blob_bins, split_layers)
from tfg_b200.structs import DATOS_MLP

pytestmark = pytest.mark.gpu

LO, HI = (-6.0, -4.0, -10.0), (6.0, 6.0, 2.0)
# small tables: dense and hashed levels, with collisions
SMALL = {"n_levels": 8, "log2_hashmap_size": 12, "base_resolution": 4.0, "per_level_scale": 2.0}


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
        d["especular"][k] = rng.uniform(0, 0.5, n)
    y = target_fn(pos, kd) if target_fn else rng.uniform(0, 2, (n, 3))
    for j, k in enumerate("rgb"):
        d["color"][k] = y[:, j]
    return d


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()


def _f16(w):
    return np.asarray(w, np.float32).astype(np.float16).astype(np.float64)


def _model(cfg, seed=3, batch=4096, table_scale=0.5):
    m = ColorMLP(batch=batch, seed=seed, encoding=HASHGRID, hashgrid=cfg)
    m.set_bounds(LO, HI)
    if table_scale:
        # table values large enough that the hash-grid features steer the output
        rng = np.random.default_rng(seed)
        m.set_table(rng.uniform(-table_scale, table_scale, m.n_table).astype(np.float32))
    return m


@pytest.mark.parametrize("cfg", [SMALL, None], ids=["small", "reference"])
def test_inference_matches_fp64_model(built, cfg):
    m = _model(cfg)
    full = {**hashgrid_reference(), **(cfg or {})}
    rng = np.random.default_rng(4)
    n = 3000
    d = _datos(rng, n)
    out = torch.zeros(n * 3, device="cuda")
    m.inference(_dev(d), out, n)
    torch.cuda.synchronize()
    got = out.view(n, 3).cpu().numpy()
    W = [_f16(w) for w in split_layers(m.get_params(WEIGHTS))]
    tab = m.get_table(WEIGHTS).astype(np.float16).astype(np.float64)   # inference reads an FP16 image
    x, _ = mo.composite_encode(mo.rows15(d, LO, HI), tab, full)
    raw = mo.forward(W, x)[0]
    want = mo.scrub(raw)
    scale = np.abs(raw).mean() + 1e-3
    err = np.abs(got - want) / scale
    assert np.isfinite(got).all()
    assert err.max() < 0.02 and err.mean() < 2e-3, (err.max(), err.mean())
    emax, emean = cache_inference_error(m, _dev(d), n, got)
    assert emax < INFER_MAX and emean < INFER_MEAN, (emax, emean)
    # the kernel's hash-grid features: the FP16 interpolation of the FP16 table image
    feat = m.encode_features(_dev(d), n).cpu().numpy().astype(np.float64)
    L2 = 2 * full["n_levels"]
    np.testing.assert_allclose(feat[:, :L2], x[:, :L2], rtol=0, atol=4e-3 * max(1.0, np.abs(x[:, :L2]).max()))
    # one-blob bins (FP32 normal CDF, then FP16) and albedos: within one FP16 step of the FP64 values
    np.testing.assert_allclose(feat[:, 32:62], mo.round_f16(x[:, 32:62]), rtol=0, atol=2.5e-4)
    # the hash-grid features matter: zero tables change the prediction
    x0 = x.copy()
    x0[:, :2 * full["n_levels"]] = 0.0
    assert np.abs(mo.forward(W, x0)[0] - raw).mean() > 10 * np.abs(got - want).mean()
    m.close()


def test_one_blob_bins_match_the_normal_cdf(built):
    # The kernels' normal CDF (Abramowitz & Stegun 26.2.17, |error| < 7.5e-8)
    # against the FP64 bins of the oracle and against CUDA's own normal CDF
    # (torch.special.ndtr in FP32) on the same FP32 inputs.
    rng = np.random.default_rng(21)
    s = np.concatenate([np.linspace(0.0, 1.0, 4097), rng.uniform(0.0, 1.0, 20000),
                        [0.0, 1.0, 1e-7, 1.0 - 6e-8, 0.125, 0.375, 0.625, 0.875]]).astype(np.float32)
    st = torch.from_numpy(s).cuda()
    got = one_blob_bins(st)
    torch.cuda.synchronize()
    g = got.cpu().numpy().astype(np.float64)
    ref = mo.one_blob(s.astype(np.float64))
    err = np.abs(g - ref).max()
    assert err < 4e-7, f"one-blob bins differ from FP64 by {err:.3e}"
    edges = torch.arange(5, device="cuda", dtype=torch.float32) / 4.0
    cdf = torch.special.ndtr((edges[None, :] - st[:, None]) * 4.0)
    cuda_bins = (cdf[:, 1:] - cdf[:, :-1]).cpu().numpy().astype(np.float64)
    assert np.abs(g - cuda_bins).max() < 5e-7
    assert (g >= -1e-7).all() and np.isfinite(g).all()
    # an empty call is a no-op
    assert one_blob_bins(torch.zeros(0, device="cuda")).shape == (0, 4)


def test_gradients_match_fp64_model(built):
    m = _model(SMALL)
    rng = np.random.default_rng(11)
    n_avail = 20000
    d = _datos(rng, n_avail)
    tab = m.get_table(WEIGHTS).astype(np.float64)
    g, gt, loss = m.compute_gradient_ex(_dev(d), n_avail, seed=5)
    idx = np.zeros(m.batch, np.int32)
    orc.cpu.orc_indices(orc.p(idx), n_avail, m.batch, 5)
    sel = d[idx]
    _, corners = mo.composite_encode(mo.rows15(sel, LO, HI), tab, SMALL)
    y = np.stack([sel["color"][k] for k in "rgb"], 1).astype(np.float64)
    # layers and tables against the model on the kernel's own FP16 operands;
    # untouched table entries get exactly zero
    check_cache_gradients(m, _dev(sel), y, g, loss, bias_col=62, g_table=gt, corners=corners,
                          table_cols=2 * SMALL["n_levels"])
    m.close()


def test_table_adam_steps_follow_the_recurrence(built):
    # Two training steps: each step's table moments, values and average against
    # the Adam / weight-average recurrence in FP64, from the tables before the
    # step and that step's gradient (same sample draw, from the step word).
    b1, b2, lr, eps, decay = 0.9, 0.99, 1e-3, 1e-15, 0.99
    m = _model(SMALL, seed=13)
    m.set_hyperparams(lr=lr, beta1=b1, beta2=b2, eps=eps, ema_decay=decay)
    rng = np.random.default_rng(17)
    n = 20000
    dd = _dev(_datos(rng, n))
    prev = [np.zeros(m.n_table) if k else m.get_table(WEIGHTS).astype(np.float64) for k in range(4)]
    for t in (1, 2):
        _, g, _ = m.compute_gradient_ex(dd, n, seed=m.state()["step"])
        g = g.astype(np.float64)
        m.train_step(dd, n, read_loss=False)
        w, e, mm, vv = [m.get_table(k).astype(np.float64) for k in range(4)]
        w0, e0, m0, v0 = prev
        m_ref = b1 * m0 + (1 - b1) * g
        v_ref = b2 * v0 + (1 - b2) * g * g
        np.testing.assert_allclose(mm, m_ref, rtol=1e-4, atol=1e-4 * np.abs(m_ref).max())
        np.testing.assert_allclose(vv, v_ref, rtol=1e-4, atol=1e-4 * np.abs(v_ref).max())
        # the value update from the device's own moments (its FP32 rounding of them)
        step = lr * (mm / (1 - b1 ** t)) / (np.sqrt(vv / (1 - b2 ** t)) + eps)
        moved = np.abs(g) > 1e-3 * np.abs(g).max()
        # the values are FP32: w0 - w carries their rounding (a few ulps of |w|)
        ulp = float(np.spacing(np.float32(np.abs(w0).max())))
        np.testing.assert_allclose((w0 - w)[moved], step[moved], rtol=1e-3, atol=4 * ulp)
        assert np.abs(w - (w0 - step)).max() < 1e-6
        np.testing.assert_allclose(e, decay * e0 + (1 - decay) * w, rtol=1e-5, atol=1e-9)
        prev = [w, e, mm, vv]
    assert m.state()["adam_t"] == 2
    m.close()


def test_online_training_fits_a_spatial_signal(built):
    def f(pos, kd):
        s = 0.5 + 0.4 * np.sin(1.3 * pos[:, 0]) * np.cos(0.9 * pos[:, 2]) + 0.2 * np.sin(2.1 * pos[:, 1])
        return np.stack([s * kd[:, 0], s * kd[:, 1], s * kd[:, 2]], 1) + 0.05

    m = ColorMLP(batch=16384, seed=8, encoding=HASHGRID)
    m.set_bounds(LO, HI)
    rng = np.random.default_rng(5)
    n = 65536
    d = _datos(rng, n, f)
    dd = _dev(d)
    first = m.train_step(dd, n)
    for _ in range(300):
        last = m.train_step(dd, n, read_loss=False)
    last = m.train_step(dd, n)
    assert np.isfinite(last) and last < 0.2 * first, (first, last)
    st = m.state()
    assert st["adam_t"] == 302
    # the tables trained: their average moved away from the initial +-1e-4
    assert np.abs(m.get_table(EMA)).max() > 1e-2
    m.close()


def test_checkpoint_round_trip(built, tmp_path):
    m = _model(SMALL, seed=9)
    rng = np.random.default_rng(6)
    d = _datos(rng, 20000)
    dd = _dev(d)
    for _ in range(5):
        m.train_step(dd, 20000, read_loss=False)
    q = _dev(_datos(rng, 1000))
    a = torch.zeros(3000, device="cuda")
    m.inference(q, a, 1000)
    path = tmp_path / "hash.ckpt"
    m.save_model(path)
    m2 = ColorMLP(batch=4096, seed=1, encoding=HASHGRID, hashgrid=SMALL)
    assert m2.load_model(path)
    b = torch.zeros(3000, device="cuda")
    m2.inference(q, b, 1000)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())
    for k in range(4):
        np.testing.assert_array_equal(m.get_table(k), m2.get_table(k))
    # a checkpoint of other tables (or of the frequency encoding) is refused
    other = ColorMLP(batch=4096, seed=1, encoding=HASHGRID, hashgrid={**SMALL, "n_levels": 7})
    assert not other.load_model(path)
    freq = ColorMLP(batch=4096, seed=1)
    assert not freq.load_model(path)
    for x in (m, m2, other, freq):
        x.close()


def test_bf16_and_fp8_inference_match_rounded_models(built):
    # BF16 and FP8 against the oracle's BF16-rounded / E4M3-quantised forward
    # passes of the same encoded inputs: the kernels' error must be of the
    # size the format itself causes.
    m = _model(SMALL, seed=12, table_scale=0.3)
    rng = np.random.default_rng(7)
    n = 4096
    d = _datos(rng, n)
    q = _dev(d)
    W = [_f16(w) for w in split_layers(m.get_params(WEIGHTS))]
    tab = m.get_table(WEIGHTS).astype(np.float16).astype(np.float64)
    x, _ = mo.composite_encode(mo.rows15(d, LO, HI), tab, SMALL)
    exact = mo.forward(W, x)[0]
    scale = np.abs(exact).mean() + 1e-3
    m.set_precision(BF16)
    b = torch.zeros(n * 3, device="cuda")
    m.inference(q, b, n)
    m.calibrate(q, n)
    m.set_precision(FP8)
    f8 = torch.zeros(n * 3, device="cuda")
    m.inference(q, f8, n)
    torch.cuda.synchronize()
    got_b, got_8 = b.view(n, 3).cpu().numpy(), f8.view(n, 3).cpu().numpy()
    ref_b = mo.scrub(mo.forward_quantized(W, x, "bf16"))
    _, hs, _ = mo.forward(W, x)
    amax = [max(1.0, float(np.abs(x[:, :62]).max()))] + [float(np.abs(h).max()) for h in hs[1:len(W)]]
    ref_8 = mo.scrub(mo.forward_quantized(W, x, "fp8", amax))
    fmt_b = np.abs(ref_b - mo.scrub(exact)).mean() / scale
    fmt_8 = np.abs(ref_8 - mo.scrub(exact)).mean() / scale
    err_b = np.abs(got_b - mo.scrub(exact)).mean() / scale
    err_8 = np.abs(got_8 - mo.scrub(exact)).mean() / scale
    assert np.isfinite(got_8).all() and np.isfinite(got_b).all()
    assert err_b < 1.5 * fmt_b + 2e-3, (err_b, fmt_b)
    assert err_8 < 1.5 * fmt_8 + 5e-3, (err_8, fmt_8)
    m.close()


def test_cache_frames_with_the_hash_grid(built):
    s = scenes.sized_terrain_scene(20000, 160, 96, 2, seed=44)
    ds = pt.DeviceScene(s, "cuda")
    params = pt.RenderParams(max_depth=6, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)
    m = ColorMLP(batch=16384, seed=5, encoding=HASHGRID)
    m.set_bounds(*s.bounds)
    r = NrcRenderer(ds, m, params, train_steps=2, max_records=8192, min_records=256, use_graph=True)
    for f in range(8):
        r.frame(f, warmup=True)
    for f in range(8, 16):
        r.frame(f, warmup=False, accumulate=True)
    r.stream.synchronize()
    img = r.mean_image().cpu().numpy()
    assert np.isfinite(img).all() and img.mean() > 0
    # 8 warm-up frames x 2 steps; the later frames' few training paths stay below min_records
    assert m.state()["adam_t"] >= 16
    m.close()
    ds.close()
