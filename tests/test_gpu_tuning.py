"""Launch tuning and the autotuners.  A tuning changes how paths are scheduled
(wavefront size, CTA size and residency, refill threshold, lanes per shadow
query), never what a path computes, so every tuning must give the same
image bit for bit -- plain passes, cache frames (eager and captured as CUDA
graphs) and the allocation-free pass.  The model autotuner must leave the
model's state untouched."""
import numpy as np
import pytest
import torch

from tfg_b200 import TfgError
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
from tfg_b200.nrc import ColorMLP, NrcRenderer
from tfg_b200.structs import DATOS_MLP

pytestmark = pytest.mark.gpu

PARAMS = pt.RenderParams(max_depth=6, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)
W, H = 160, 96
N = W * H


@pytest.fixture(scope="module")
def scene(built):
    s = scenes.sized_terrain_scene(20000, W, H, 3, seed=41)
    ds = pt.DeviceScene(s, "cuda")
    yield s, ds
    ds.close()


@pytest.fixture(autouse=True)
def default_tuning():
    pt.set_tuning(pt.RenderTuning.default())
    yield
    pt.set_tuning(pt.RenderTuning.default())


def _render(ds, spp=4, frame=9):
    p = pt.RenderParams(**{**PARAMS.__dict__, "spp": spp, "accumulate": 1})
    img = torch.zeros(N * 3, dtype=torch.float32, device="cuda")
    acc = torch.zeros(N * 3, dtype=torch.float32, device="cuda")
    pt.render_pass(ds, p, frame, img, acc)
    torch.cuda.synchronize()
    return img.cpu().numpy(), acc.cpu().numpy()


TUNINGS = [
    pt.RenderTuning(wavefront_paths=1024),               # 15 chunks per sample
    pt.RenderTuning(wavefront_paths=5003),               # chunks that straddle samples
    pt.RenderTuning(wavefront_paths=N // 2),
    pt.RenderTuning(wavefront_paths=2 * N),              # two samples per wavefront
    pt.RenderTuning(wavefront_paths=3 * N + 7),          # ragged multi-sample wavefronts
    pt.RenderTuning(wavefront_paths=8 * N),              # the whole call in one wavefront
    pt.RenderTuning(trace_threads=64),
    pt.RenderTuning(trace_threads=256),
    pt.RenderTuning(trace_warps_per_sm=8),
    pt.RenderTuning(refill_min=1),
    pt.RenderTuning(refill_min=32),
    pt.RenderTuning(shadow_one_lane=1),
    pt.RenderTuning(refill_min_primary=32),
    pt.RenderTuning(refill_min_primary=2, refill_min=29),
    pt.RenderTuning(overlap_shadow=0),
    pt.RenderTuning(overlap_shadow=0, wavefront_paths=2 * N),
    pt.RenderTuning(overlap_shadow=1, wavefront_paths=3 * N + 7, trace_threads=64, shadow_one_lane=1),
    pt.RenderTuning(wavefront_paths=2 * N + 1000, trace_threads=256, trace_warps_per_sm=16, refill_min=12,
                    shadow_one_lane=1),
]


def test_every_tuning_renders_the_same_image(scene):
    _, ds = scene
    want_img, want_acc = _render(ds)
    assert np.isfinite(want_acc).all() and want_acc.max() > 0
    for t in TUNINGS:
        pt.set_tuning(t)
        assert pt.get_tuning() == t
        img, acc = _render(ds)
        np.testing.assert_array_equal(img, want_img, err_msg=str(t))
        np.testing.assert_array_equal(acc, want_acc, err_msg=str(t))


def test_reference_triangles_and_profile_counts_under_tuning(scene):
    # the reference triangle layout and the counting kernel variants take the
    # same tuned launch shapes
    _, ds = scene
    p = pt.RenderParams(**{**PARAMS.__dict__, "tri_format": pt.TRIS_REF, "spp": 2, "accumulate": 1,
                           "profile": pt.PROFILE_COUNTS})
    outs = []
    for t in (pt.RenderTuning.default(), pt.RenderTuning(wavefront_paths=4096, trace_threads=64, shadow_one_lane=1)):
        pt.set_tuning(t)
        pt.profile_reset()
        acc = torch.zeros(N * 3, dtype=torch.float32, device="cuda")
        pt.render_pass(ds, p, 3, None, acc)
        prof = pt.profile_get()
        outs.append((acc.cpu().numpy(), prof["rays"], prof["shadow_rays"], prof["nodes"]))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    assert outs[0][1:] == outs[1][1:]          # the same rays, shadow rays and nodes


def test_static_pass_under_tuning(built):
    s = scenes.box_icosphere(64, 48, subdiv=3)
    ds = pt.DeviceScene(s, "cuda")
    p = pt.RenderParams(max_depth=5, rr_min_depth=3, shadow_mesh=1, spp=3, accumulate=1)
    n = 64 * 48
    acc0 = torch.zeros(n * 3, device="cuda")
    pt.render_pass(ds, p, 5, None, acc0)
    for t in (pt.RenderTuning(wavefront_paths=1024), pt.RenderTuning(wavefront_paths=4 * n, trace_threads=256)):
        pt.set_tuning(t)
        acc = torch.zeros(n * 3, device="cuda")
        pt.render_pass_static(ds, p, 5, None, acc)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(acc.cpu().numpy(), acc0.cpu().numpy())
    ds.close()


@pytest.mark.parametrize("graph", [False, True])
def test_cache_frames_under_tuning(scene, graph):
    # Cache passes split a sample into wavefronts but never merge samples.
    # Without training steps a frame is a function of the model and the
    # frame number.  With graphs, a tuning change re-captures the frame.
    s, ds = scene

    def frames(tunings):
        m = ColorMLP(batch=16384, seed=5)
        m.set_bounds(*s.bounds)
        r = NrcRenderer(ds, m, PARAMS, train_steps=0, max_records=4096, min_records=256, use_graph=graph)
        out = []
        for f, t in zip((6, 7, 8), tunings):
            pt.set_tuning(t)
            r.frame(f, warmup=False, accumulate=False)
            r.stream.synchronize()
            out.append(r.image().cpu().numpy().copy())
        m.close()
        return out

    d = pt.RenderTuning.default()
    want = frames([d, d, d])
    got = frames([pt.RenderTuning(wavefront_paths=4000, overlap_shadow=1),
                  pt.RenderTuning(wavefront_paths=4 * N, trace_threads=64),
                  pt.RenderTuning(wavefront_paths=N // 3, shadow_one_lane=1, refill_min=3, overlap_shadow=1)])
    for g, w in zip(got, want):
        assert np.isfinite(g).all()
        np.testing.assert_array_equal(g, w)


def test_bad_tunings_are_rejected(built):
    for bad in (pt.RenderTuning(wavefront_paths=100), pt.RenderTuning(wavefront_paths=(1 << 26) + 1),
                pt.RenderTuning(trace_threads=96), pt.RenderTuning(refill_min=0), pt.RenderTuning(refill_min=33),
                pt.RenderTuning(trace_warps_per_sm=-1), pt.RenderTuning(shadow_one_lane=2),
                pt.RenderTuning(refill_min_primary=33), pt.RenderTuning(overlap_shadow=2)):
        with pytest.raises(TfgError):
            pt.set_tuning(bad)
    assert pt.get_tuning() == pt.RenderTuning.default()


def test_autotune_picks_a_measured_tuning(scene):
    _, ds = scene
    want_img, want_acc = _render(ds)
    best, table = pt.autotune(ds, PARAMS, repeats=2)
    assert pt.get_tuning() == best
    assert len(table) >= 15
    assert all(ms > 0 for _, ms in table)
    tried = [t for t, _ in table]
    assert best in tried
    # the winner is within 1% of the fastest candidate seen, or faster than the start
    best_ms = min(ms for t, ms in table if t == best)
    assert best_ms <= table[0][1] + 1e-6
    img, acc = _render(ds)
    np.testing.assert_array_equal(acc, want_acc)
    np.testing.assert_array_equal(img, want_img)


def _random_queries(n, seed):
    rng = np.random.default_rng(seed)
    d = np.zeros(n, DATOS_MLP)
    for f in ("posicion", "direccion", "normal"):
        for c in "xyz":
            d[f][c] = rng.uniform(0.0, 1.0, n)
    for f in ("difuso", "especular", "color"):
        for c in "rgb":
            d[f][c] = rng.uniform(0.0, 1.0, n)
    return torch.from_numpy(d.view(np.uint8).copy()).cuda()


def test_mlp_autotune_leaves_the_model_as_it_was(built):
    m = ColorMLP(batch=16384, seed=21)
    m.set_bounds((0, 0, 0), (1, 1, 1))
    train = _random_queries(20000, 1)
    for _ in range(3):
        m.train_step(train, 20000)
    n = 100000
    q = _random_queries(n, 2)
    out0 = torch.zeros(n * 3, device="cuda")
    m.inference(q, out0, n)
    g0, _ = m.compute_gradient(train, 20000, seed=77)
    before = [m.get_params(k) for k in range(4)]
    state = m.state()
    res = m.autotune(q, torch.zeros(n * 3, device="cuda"), n, repeats=3)
    assert res["wgrad_ms"] > 0 and res["infer_ms"] > 0
    assert m.get_tuning() == {"wgrad_tiles_per_cta": res["wgrad_tiles_per_cta"], "infer_ctas": res["infer_ctas"]}
    for k in range(4):
        np.testing.assert_array_equal(m.get_params(k), before[k])
    assert m.state() == state
    # inference rows do not depend on the grid; gradients only up to the order
    # of FP32 additions
    out1 = torch.zeros(n * 3, device="cuda")
    m.inference(q, out1, n)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out1.cpu().numpy(), out0.cpu().numpy())
    g1, _ = m.compute_gradient(train, 20000, seed=77)
    np.testing.assert_allclose(g1, g0, rtol=1e-4, atol=1e-6 * np.abs(g0).max())
    m.close()


@pytest.mark.parametrize("tiles", [1, 3, 64, 200])
def test_mlp_gradient_under_tiling(built, tiles):
    m = ColorMLP(batch=16384, seed=22)
    m.set_bounds((0, 0, 0), (1, 1, 1))
    train = _random_queries(30000, 3)
    g0, l0 = m.compute_gradient(train, 30000, seed=5)
    m.set_tuning(wgrad_tiles_per_cta=tiles, infer_ctas=37)
    g1, l1 = m.compute_gradient(train, 30000, seed=5)
    assert l1 == pytest.approx(l0, rel=1e-5)
    np.testing.assert_allclose(g1, g0, rtol=1e-4, atol=1e-6 * np.abs(g0).max())
    m.close()
