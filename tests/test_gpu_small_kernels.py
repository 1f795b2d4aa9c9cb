"""The element-wise kernels around the cache (composite, targets, tail
queries, batch indices, feature rows, output scrub, default camera) must be
bit-identical to the reference's own kernels (oracle/_ref) and to the CPU
restatement on the same random inputs, including NaN / Inf / negative /
huge values and invalid records."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from tfg_b200 import _lib
from tfg_b200.structs import BOUNDS, CAMARA, COLOR, DATOS_MLP, REGISTRO

pytestmark = pytest.mark.gpu


def _ref():
    r = orc.ref()
    if r is None:
        pytest.skip("reference kernels (oracle/_ref) not built")
    return r


def _dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()


def _host(t: torch.Tensor, dtype) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy().view(dtype)


def _rand_colors(rng, n, special=True):
    c = rng.uniform(-0.5, 3.0, (n, 3)).astype(np.float32)
    if special:
        c[rng.random((n, 3)) < 0.03] = np.nan
        c[rng.random((n, 3)) < 0.03] = np.inf
        c[rng.random((n, 3)) < 0.03] = -np.inf
        c[rng.random((n, 3)) < 0.03] = 3e5
    return c


def _datos(rng, n):
    d = np.zeros(n, DATOS_MLP)
    for f in ("posicion", "direccion", "normal"):
        v = rng.uniform(-8, 8, (n, 3))
        d[f]["x"], d[f]["y"], d[f]["z"] = v.T
    for f in ("difuso", "especular", "color"):
        c = _rand_colors(rng, n, special=(f == "color"))
        d[f]["r"], d[f]["g"], d[f]["b"] = c.T
    return d


def _regs(rng, n):
    r = np.zeros(n, REGISTRO)
    for part in ("head", "tail"):
        for f in ("posicion", "direccion", "normal"):
            v = rng.uniform(-5, 5, (n, 3))
            r[part][f]["x"], r[part][f]["y"], r[part][f]["z"] = v.T
        for f in ("difuso", "especular"):
            c = rng.uniform(0, 1, (n, 3)).astype(np.float32)
            r[part][f]["r"], r[part][f]["g"], r[part][f]["b"] = c.T
    for f in ("luz_acumulada_sufijo", "throughput_sufijo", "factor_normalizacion"):
        c = _rand_colors(rng, n)
        r[f]["r"], r[f]["g"], r[f]["b"] = c.T
    r["factor_normalizacion"]["r"][rng.random(n) < 0.05] = 0.0
    r["valido"] = (rng.random(n) < 0.8).astype(np.uint8)
    return r


def _bounds():
    b = np.zeros(1, BOUNDS)
    b["min"]["x"], b["min"]["y"], b["min"]["z"] = -6.0, -4.0, -10.0
    b["max"]["x"], b["max"]["y"], b["max"]["z"] = 6.0, 6.0, 2.0
    return b


def test_composite_bit_exact():
    rng = np.random.default_rng(1)
    W, H = 48, 32
    img, pred, thr = (_rand_colors(rng, W * H, special=False) for _ in range(3))
    thr[rng.random(W * H) < 0.3] = 0.0
    a, b = _dev(img), _dev(img)
    p, t = _dev(pred), _dev(thr)
    _lib.call("tfgLaunchKernelComposite", a.data_ptr(), p.data_ptr(), t.data_ptr(), W, H, None)
    assert _ref().ref_composite(b.data_ptr(), p.data_ptr(), t.data_ptr(), W, H) == 0
    ga, gb = _host(a, np.uint32), _host(b, np.uint32)
    assert np.array_equal(ga, gb)
    c = img.copy()
    orc.cpu.orc_composite(orc.p(c), orc.p(pred), orc.p(thr), W * H)
    # the oracle rounds the multiply and the add separately; the device fuses them
    assert np.allclose(ga.view(np.float32).reshape(-1, 3), c, rtol=1e-6, atol=1e-6)


def test_targets_and_tail_bit_exact():
    rng = np.random.default_rng(2)
    n = 5000
    regs = _regs(rng, n)
    tail = _rand_colors(rng, n, special=False)
    dr, dt = _dev(regs), _dev(tail)
    oa = _dev(np.zeros(n, DATOS_MLP))
    ob = _dev(np.zeros(n, DATOS_MLP))
    _lib.call("tfgLaunchKernelCalcularTargets", dr.data_ptr(), dt.data_ptr(), oa.data_ptr(), n, None)
    assert _ref().ref_targets(dr.data_ptr(), dt.data_ptr(), ob.data_ptr(), n) == 0
    assert np.array_equal(_host(oa, np.uint8), _host(ob, np.uint8))
    c = np.zeros(n, DATOS_MLP)
    orc.cpu.orc_targets(orc.p(regs), orc.p(tail), orc.p(c), n)
    got = _host(oa, DATOS_MLP)
    for f in "rgb":
        np.testing.assert_allclose(got["color"][f], c["color"][f], rtol=1e-5, atol=1e-5)
    ta = _dev(np.zeros(n, DATOS_MLP))
    tb = _dev(np.zeros(n, DATOS_MLP))
    _lib.call("tfgLaunchKernelPrepararInferenciaTail", dr.data_ptr(), ta.data_ptr(), n, None)
    assert _ref().ref_tail(dr.data_ptr(), tb.data_ptr(), n) == 0
    assert np.array_equal(_host(ta, np.uint8), _host(tb, np.uint8))


def test_indices_rows_scrub_bit_exact():
    rng = np.random.default_rng(3)
    n, batch = 7000, 4096
    d = _datos(rng, n)
    dd = _dev(d)
    ia = torch.zeros(batch, dtype=torch.int32, device="cuda")
    ib = torch.zeros(batch, dtype=torch.int32, device="cuda")
    _lib.call("tfgLaunchGenerarIndicesAleatorios", ia.data_ptr(), n, batch, 12345, None)
    assert _ref().ref_indices(ib.data_ptr(), n, batch, 12345) == 0
    assert torch.equal(ia, ib)
    ci = np.zeros(batch, np.int32)
    orc.cpu.orc_indices(orc.p(ci), n, batch, 12345)
    assert np.array_equal(ia.cpu().numpy(), ci)

    b = _bounds()
    bb = b.ctypes.data
    ina = torch.zeros(batch * 15, device="cuda")
    inb = torch.zeros(batch * 15, device="cuda")
    tga = torch.zeros(batch * 3, device="cuda")
    tgb = torch.zeros(batch * 3, device="cuda")
    _lib.call("tfgLaunchPrepararDatosEntrenamiento", dd.data_ptr(), ia.data_ptr(), batch, 15, 3, bb,
              ina.data_ptr(), tga.data_ptr(), None)
    assert _ref().ref_train_rows(dd.data_ptr(), ia.data_ptr(), batch, 15, 3, bb, inb.data_ptr(), tgb.data_ptr()) == 0
    torch.cuda.synchronize()
    assert torch.equal(ina.view(torch.int32), inb.view(torch.int32))
    assert torch.equal(tga.view(torch.int32), tgb.view(torch.int32))
    ci_in, ci_t = np.zeros(batch * 15, np.float32), np.zeros(batch * 3, np.float32)
    orc.cpu.orc_train_rows(orc.p(d), orc.p(ci), batch, 15, 3, bb, orc.p(ci_in), orc.p(ci_t))
    assert np.array_equal(ina.cpu().numpy().view(np.uint32), ci_in.view(np.uint32))

    fa = torch.zeros(n * 15, device="cuda")
    fb = torch.zeros(n * 15, device="cuda")
    _lib.call("tfgLaunchPrepararDatosInferencia", dd.data_ptr(), n, 15, fa.data_ptr(), bb, None)
    assert _ref().ref_infer_rows(dd.data_ptr(), n, 15, fb.data_ptr(), bb) == 0
    torch.cuda.synchronize()
    assert torch.equal(fa.view(torch.int32), fb.view(torch.int32))

    net = _rand_colors(rng, n).reshape(-1)
    dn = torch.from_numpy(net.copy()).cuda()
    sa = _dev(np.zeros(n, COLOR))
    sb = _dev(np.zeros(n, COLOR))
    _lib.call("tfgLaunchGuardarSalidaInferencia", dn.data_ptr(), sa.data_ptr(), n, None)
    assert _ref().ref_scrub(dn.data_ptr(), sb.data_ptr(), n) == 0
    assert np.array_equal(_host(sa, np.uint8), _host(sb, np.uint8))
    co = np.zeros(n, COLOR)
    orc.cpu.orc_scrub(orc.p(net), orc.p(co), n)
    assert np.array_equal(_host(sa, np.uint8), co.view(np.uint8))


@pytest.mark.parametrize("wh", [(512, 512), (1920, 1080), (7, 3)])
def test_default_camera_bit_exact(wh):
    W, H = wh
    a = torch.zeros(112, dtype=torch.uint8, device="cuda")
    b = torch.zeros(112, dtype=torch.uint8, device="cuda")
    _lib.call("tfgLaunchInicializarCamara", a.data_ptr(), W, H, None)
    assert _ref().ref_camera(b.data_ptr(), W, H) == 0
    assert torch.equal(a, b)
    c = np.zeros(1, CAMARA)
    orc.cpu.orc_default_camera(orc.p(c), W, H)
    got = a.cpu().numpy().view(CAMARA)
    for f in ("posicion", "frente", "arriba", "izquierda"):
        for k in "xyz":
            assert got[f][k] == c[f][k]
    assert abs(float(got["alto_plano"][0]) - float(c["alto_plano"][0])) <= 1e-6
