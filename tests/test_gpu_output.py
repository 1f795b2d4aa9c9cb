"""Final-image and reconstruction entry points on the GPU: the filmic tone
map matches the CPU restatement bit for bit; tfgNrcReconstruct equals the
reference's sample loop built from the single-step entry points; a cache
checkpoint restores the model exactly."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
from tfg_b200.nrc import EMA, WEIGHTS, ADAM_M, ADAM_V, ColorMLP, NrcRenderer, reconstruct
from tfg_b200.structs import DATOS_MLP

pytestmark = pytest.mark.gpu

PARAMS = pt.RenderParams(max_depth=6, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)


@pytest.fixture(scope="module")
def trained(built):
    s = scenes.spheres_terrain(96, 64, subdiv=2, terrain_n=40)
    ds = pt.DeviceScene(s, "cuda")
    m = ColorMLP(batch=4096, seed=5)
    m.set_bounds(*s.bounds)
    r = NrcRenderer(ds, m, PARAMS, train_steps=2, max_records=8192, min_records=256)
    for f in range(12):
        r.frame(f, warmup=f < 8, accumulate=False)
    r.stream.synchronize()
    yield s, ds, m
    m.close()
    ds.close()


def test_tonemap_matches_cpu_restatement(built):
    rng = np.random.default_rng(3)
    W, H, frames = 97, 33, 7
    s = (rng.lognormal(0.0, 1.5, (H * W * 3)) * frames).astype(np.float32)
    s[:5] = [0.0, 1e9, 0.5, 3.0, 1e-7]
    hdr, rgb8 = pt.tonemap_filmic(torch.from_numpy(s).cuda(), frames, W, H)
    torch.cuda.synchronize()
    want_hdr = np.zeros_like(s)
    want_b = np.zeros(s.size, np.uint8)
    orc.cpu.orc_tonemap_filmic(orc.p(s), frames, W * H, orc.p(want_hdr), orc.p(want_b))
    np.testing.assert_array_equal(hdr.cpu().numpy().reshape(-1), want_hdr)
    np.testing.assert_array_equal(rgb8.cpu().numpy().reshape(-1), want_b)


def test_reconstruction_equals_the_sample_loop(trained):
    s, ds, m = trained
    W, H = s.width, s.height
    n = W * H
    spp = 3
    got = reconstruct(ds, m, PARAMS, spp, first_frame=100)
    # the reference's loop: render with cache queries, infer + composite, add
    img = torch.zeros(n * 3, device="cuda")
    acc = torch.zeros(n * 3, device="cuda")
    buf = pt.NrcBuffers(n, "cuda")
    for k in range(spp):
        pt.render_pass(ds, PARAMS, 100 + k, img, nrc=buf, use_inf=True, train=False)
        m.inference_composite(buf.infer, buf.thr, img, n)
        acc += img
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.cpu().numpy(), acc.cpu().numpy())
    hdr, rgb8 = pt.tonemap_filmic(got, spp, W, H)
    assert np.isfinite(hdr.cpu().numpy()).all() and rgb8.cpu().numpy().max() > 0


def test_checkpoint_round_trip(trained, tmp_path):
    s, ds, m = trained
    path = tmp_path / "cache.tfgnrc"
    m.save_model(path)
    m2 = ColorMLP(batch=4096, seed=99)
    assert m2.load_model(path)
    for which in (WEIGHTS, EMA, ADAM_M, ADAM_V):
        np.testing.assert_array_equal(m2.get_params(which), m.get_params(which))
    assert m2.state() == m.state()
    rng = np.random.default_rng(1)
    n = 1000
    d = np.zeros(n, DATOS_MLP)
    lo, hi = s.bounds
    for j, k in enumerate("xyz"):
        d["posicion"][k] = rng.uniform(lo[j], hi[j], n)
        d["normal"][k] = rng.uniform(0, 1, n)
        d["direccion"][k] = rng.uniform(0, 1, n)
    dd = torch.from_numpy(d.view(np.uint8).copy()).cuda()
    a, b = torch.zeros(n * 3, device="cuda"), torch.zeros(n * 3, device="cuda")
    m.inference(dd, a, n)
    m2.inference(dd, b, n)           # bounds came from the checkpoint
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())
    m2.close()
    deeper = ColorMLP(batch=4096, seed=1, hidden_layers=7)
    assert not deeper.load_model(path)     # depth mismatch is refused
    assert not deeper.load_model(tmp_path / "missing.tfgnrc")
    deeper.close()
