"""Online radiance caching end to end on the GPU (tfgNrcFrame): frames run
without host synchronisation (optionally as a replayed CUDA graph), the cache
trains on the path suffixes the tracer generates, and a cache-assisted 1-spp
frame beats plain path tracing given the same GPU time, both scored by
relMSE against a high-spp plain path-traced reference accumulated in FP64."""
import numpy as np
import pytest
import torch

from tests.helpers import rel_mse
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
from tfg_b200.nrc import BF16, FP16, ColorMLP, NrcRenderer

pytestmark = pytest.mark.gpu

PARAMS = pt.RenderParams(max_depth=8, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)


def reference_image(ds, spp, first_frame=1_000_000, batch=64):
    """Mean of `spp` samples: FP32 sums of `batch` samples added in FP64."""
    tot = np.zeros((ds.scene.height, ds.scene.width, 3))
    for b in range(spp // batch):
        img = pt.accumulate_spp(ds, PARAMS, batch, first_frame + b * batch)
        torch.cuda.synchronize()
        tot += img.cpu().numpy().astype(np.float64)
    return tot / (spp // batch)


@pytest.fixture(scope="module")
def scene_ds(built):
    s = scenes.spheres_terrain(320, 176, subdiv=4, terrain_n=160)
    ds = pt.DeviceScene(s, "cuda")
    yield s, ds
    ds.close()


def _mlp(scene):
    m = ColorMLP(batch=16384, seed=42)
    m.set_bounds(*scene.bounds)
    return m


def test_graph_replay_matches_eager(scene_ds):
    s, ds = scene_ds
    imgs = []
    for graph in (False, True):
        m = _mlp(s)
        r = NrcRenderer(ds, m, PARAMS, train_steps=1, use_graph=graph)
        r.frame(5, warmup=False, accumulate=False)
        r.stream.synchronize()
        imgs.append(r.image().cpu().numpy().copy())
        m.close()
    assert np.isfinite(imgs[0]).all()
    np.testing.assert_array_equal(imgs[0], imgs[1])


def test_precision_change_recaptures_the_frame_graph(scene_ds):
    # The inference precision is part of a captured frame's identity: after
    # switching it, a replayed frame must match the same frame run eagerly.
    s, ds = scene_ds
    imgs = {}
    for graph in (False, True):
        m = _mlp(s)
        r = NrcRenderer(ds, m, PARAMS, train_steps=0, use_graph=graph)
        r.frame(5, accumulate=False)                 # FP16 (captured when graph)
        m.set_precision(BF16)
        r.frame(5, accumulate=False)
        r.stream.synchronize()
        imgs[graph] = r.image().cpu().numpy().copy()
        m.set_precision(FP16)
        r.frame(5, accumulate=False)
        r.stream.synchronize()
        imgs[(graph, "fp16")] = r.image().cpu().numpy().copy()
        m.close()
    np.testing.assert_array_equal(imgs[True], imgs[False])
    np.testing.assert_array_equal(imgs[(True, "fp16")], imgs[(False, "fp16")])
    assert not np.array_equal(imgs[False], imgs[(False, "fp16")])


def test_frames_train_the_cache(scene_ds):
    s, ds = scene_ds
    m = _mlp(s)
    r = NrcRenderer(ds, m, PARAMS, train_steps=4)
    for f in range(6):
        r.frame(f, warmup=True)
    r.stream.synchronize()
    st = m.state()
    # warm-up frames make every pixel a training path: plenty of records, 4 steps each
    assert st["adam_t"] == 24 and st["step"] == 24
    assert st["records"] == min(65536, (s.width * s.height) // 4 * 4) or st["records"] > 1024
    assert np.isfinite(st["loss_ema"]) and st["loss_ema"] > 0
    m.close()


@pytest.fixture(scope="module")
def reference_1024(scene_ds):
    return reference_image(scene_ds[1], 1024)


# footprint 0.01: the reference's policy (render.h:86-102), which answers only
# the paths whose footprint has grown; 0: every path ends into the cache at its
# first diffuse vertex, the primary hit included, which removes the noise of
# every later bounce and is the policy the 2x target is measured with.
@pytest.mark.parametrize("footprint,min_ratio", [(0.01, 1.0), (0.0, 2.0)])
def test_cache_beats_plain_path_tracing_at_equal_time(scene_ds, reference_1024, footprint, min_ratio):
    s, ds = scene_ds
    ref = reference_1024
    m = _mlp(s)
    r = NrcRenderer(ds, m, PARAMS, train_steps=4, footprint=footprint)
    frame = 0
    for _ in range(48):                   # reference warm-up (main.cpp:946)
        r.frame(frame, warmup=True, accumulate=False)
        frame += 1
    for _ in range(80):
        r.frame(frame, accumulate=False)
        frame += 1
    r.stream.synchronize()
    # GPU time of one cache frame (render + inference + training) vs one plain pass
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(r.stream)
    for _ in range(10):
        r.frame(frame, accumulate=False)
        frame += 1
    e1.record(r.stream)
    e1.synchronize()
    t_nrc = e0.elapsed_time(e1) / 10
    nrc_img = r.image().cpu().numpy().astype(np.float64)
    img = torch.zeros(s.width * s.height * 3, device="cuda")
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    for k in range(10):
        pt.render_pass(ds, PARAMS, 500 + k, img)
    p1.record()
    p1.synchronize()
    t_pt = p0.elapsed_time(p1) / 10
    spp_equal = max(1, int(round(t_nrc / t_pt)))
    plain = pt.accumulate_spp(ds, PARAMS, spp_equal, 7000).cpu().numpy().astype(np.float64)
    bad = {k: int((~np.isfinite(v)).sum()) for k, v in (("ref", ref), ("nrc", nrc_img), ("plain", plain))}
    assert not any(bad.values()), f"non-finite pixels: {bad}"
    e_nrc, e_pt = rel_mse(nrc_img, ref), rel_mse(plain, ref)
    # plain path tracing is unbiased: its relMSE scales as 1 / time, so the
    # equal-time comparison is the ratio of relMSE x time
    eff = (e_pt * t_pt * spp_equal) / (e_nrc * t_nrc)
    print(f"nrc frame {t_nrc:.3f} ms, plain pass {t_pt:.3f} ms -> {spp_equal} spp; relMSE nrc {e_nrc:.4f} "
          f"plain {e_pt:.4f} ratio {e_pt / e_nrc:.2f}, relMSE x time ratio {eff:.2f}")
    assert np.isfinite(nrc_img).all()
    assert e_pt / e_nrc > min_ratio and eff > min_ratio, (e_nrc, e_pt, eff)
    m.close()
