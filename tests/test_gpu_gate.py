"""The radiance cache's per-cell gate, judged by the path tracer.

Training records whose suffix ran to its end are unbiased one-sample
estimates of what the cache should answer at their head.  Each frame the
gate compares the cache's answer there with them, per cell of a grid over
the scene bounds, and a path may end into the cache (the query decision of
render.h:182), record a bootstrapped head or cut its suffix only in a cell
whose running relative error is below the threshold.

* threshold 0: the gate is off and the frame is the reference's frame
  (render + cache answers composited), bit for bit;
* a vanishing threshold: no cell ever opens, no query is answered, and every
  frame is plain path tracing on the same random numbers, bit for bit;
* the camera moves into a region no path has seen: almost no query is
  answered there (under a quarter of what the judged room answered) until
  the gate has seen the cache be right there, then it opens;
* the lighting changes under a trained cache: the gate closes within a few
  frames, and opens again once the lighting is back.
"""
import numpy as np
import pytest
import torch

from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
from tfg_b200.nrc import ColorMLP, NrcRenderer
from tfg_b200.scenes import Scene

pytestmark = pytest.mark.gpu

PARAMS = pt.RenderParams(max_depth=8, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)


@pytest.fixture(scope="module")
def terrain(built):
    s = scenes.spheres_terrain(320, 176, subdiv=4, terrain_n=160)
    ds = pt.DeviceScene(s, "cuda")
    yield s, ds
    ds.close()


def _mlp(scene, seed=42):
    m = ColorMLP(batch=16384, seed=seed)
    m.set_bounds(*scene.bounds)
    return m


def _frame_image(r, f):
    r.frame(f, accumulate=False)
    r.stream.synchronize()
    return r.image().cpu().numpy().copy()


# The gate learns from the frame's training records, and neither it nor the
# training runs below `min_records` records: these small frames trace a
# quarter of their paths for training so that every frame has enough.


def _answered(r):
    """Pixels whose value includes a cache answer (non-zero query throughput)."""
    return float((r.thr.view(-1, 3) != 0).any(dim=1).float().mean())


def test_threshold_zero_is_the_reference_frame(terrain):
    s, ds = terrain
    W, H = s.width, s.height
    n = W * H
    m = _mlp(s)
    r = NrcRenderer(ds, m, PARAMS, train_steps=0, gate_threshold=0.0, use_graph=False)
    got = _frame_image(r, 17)
    # the same frame from the single-step entries: render with cache queries
    # and training records (tfgRenderPass), then answer and composite them
    nb = pt.NrcBuffers(n, "cuda")
    img = torch.zeros(n * 3, dtype=torch.float32, device="cuda")
    pt.render_pass(ds, PARAMS, 17, img, nrc=nb, use_inf=True, train=True)
    m.inference_composite(nb.infer, nb.thr, img, n)
    torch.cuda.synchronize()
    want = img.view(H, W, 3).cpu().numpy()
    assert np.isfinite(got).all()
    diff = got.view(np.uint32) != want.view(np.uint32)
    assert not diff.any(), f"{int(diff.any(axis=2).sum())} pixels differ"
    assert _answered(r) > 0.02, _answered(r)
    m.close()


def test_vanishing_threshold_renders_plain_path_tracing(terrain):
    s, ds = terrain
    W, H = s.width, s.height
    m = _mlp(s)
    r = NrcRenderer(ds, m, PARAMS, train_steps=4, gate_threshold=1e-30, use_graph=True)
    for f in range(3):
        r.frame(f, warmup=True, accumulate=False)
    img = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    for f in (3, 4, 5, 6):
        got = _frame_image(r, f)
        pt.render_pass(ds, PARAMS, f, img)
        torch.cuda.synchronize()
        want = img.view(H, W, 3).cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"frame {f}"
        assert _answered(r) == 0.0
    st = m.state()
    assert st["gate"] == 0 and st["adam_t"] > 0   # the cache trained, the gate never opened
    m.close()


def two_rooms(width=160, height=96, offset=20.0) -> Scene:
    """Two closed boxes `offset` apart along x, each with a displaced
    icosphere and a point light: no path leaves the box it starts in."""
    rng = np.random.default_rng(5)
    Vs, Fs, kds, boxes = [], [], [], []
    off = 0
    for k in range(2):
        dx = k * offset
        V, F = scenes.displaced_icosphere(3, (dx, -0.8, -0.6), 1.0, 0.1, 11 + k)
        Vs.append(V)
        Fs.append(F + off)
        off += len(V)
        kds.append(np.repeat(rng.uniform(0.2, 0.8, size=(1, 3)), len(F), axis=0))
        boxes.append(scenes.box_prims((dx - 2.6, -2.0, -4.0), (dx + 2.6, 2.4, 5.5),
                                      {"left": (0.7, 0.2, 0.2), "right": (0.2, 0.7, 0.2)}))
    mesh = scenes.mesh_prims(np.concatenate(Vs), np.concatenate(Fs), np.concatenate(kds).astype(np.float32))
    L = scenes.lights(((0.0, 1.9, 0.8), (25.0, 25.0, 25.0)), ((offset, 1.9, 0.8), (25.0, 25.0, 25.0)))
    cam = room_camera(0, width, height, offset)
    return Scene(np.concatenate(boxes), mesh, L, cam, width, height,
                 bounds=((-2.6, -2.0, -4.0), (offset + 2.6, 2.4, 5.5)), name="two_rooms")


def room_camera(k, width, height, offset=20.0):
    dx = k * offset
    return scenes.make_camera((dx, -0.75, 4.25), (dx, -0.75, 0.0), width=width, height=height)


def test_gate_stays_closed_in_an_unseen_region_until_judged(built):
    s = two_rooms()
    ds = pt.DeviceScene(s, "cuda")
    m = _mlp(s, seed=3)
    r = NrcRenderer(ds, m, PARAMS, train_steps=4, gate_threshold=0.5, use_graph=True, min_records=64,
                    train_fraction=0.25)
    f = 0
    for _ in range(8):
        r.frame(f, warmup=True, accumulate=False)
        f += 1
    for _ in range(24):
        r.frame(f, accumulate=False)
        f += 1
    r.stream.synchronize()
    open_a = m.state()["gate"]
    seen = _answered(r)
    assert open_a > 0 and seen > 0.02, (open_a, seen)
    # into the other room: nothing there has been judged yet
    ds.set_camera(room_camera(1, s.width, s.height))
    r.frame(f, accumulate=False)
    f += 1
    r.stream.synchronize()
    first = _answered(r)
    assert first < 0.25 * seen, (first, seen)
    answered = [first]
    for _ in range(24):
        r.frame(f, accumulate=False)
        f += 1
        r.stream.synchronize()
        answered.append(_answered(r))
    # the new room's cells open once judged; the old room's close as their
    # evidence decays away (no new samples there)
    assert max(answered[-4:]) > max(5.0 * first, 0.05) and m.state()["gate"] > 0, (
        answered[::4], open_a, m.state()["gate"])
    m.close()
    ds.close()


def test_gate_closes_when_the_lighting_changes(terrain):
    s, ds = terrain
    m = _mlp(s, seed=9)
    r = NrcRenderer(ds, m, PARAMS, train_steps=4, gate_threshold=0.5, use_graph=True, min_records=64,
                    train_fraction=0.25)
    f = 0
    for _ in range(8):
        r.frame(f, warmup=True, accumulate=False)
        f += 1
    for _ in range(24):
        r.frame(f, accumulate=False)
        f += 1
    r.stream.synchronize()
    open0 = m.state()["gate"]
    answered0 = _answered(r)
    assert open0 > 50 and answered0 > 0.02, (open0, answered0)
    # freeze the cache, then make the lights 50x brighter: its answers are now
    # far too dark (relative error ~1 against the new targets)
    r.cfg.train_steps = 0
    lights0 = ds.lights.clone()
    bright = s.lights.copy()
    for k in ("r", "g", "b"):
        bright["intensidad"][k] *= 50.0
    ds.lights.copy_(torch.from_numpy(bright.view(np.uint8).copy()).cuda())
    torch.cuda.synchronize()
    counts = []
    for _ in range(6):
        r.frame(f, accumulate=False)
        f += 1
        r.stream.synchronize()
        counts.append(m.state()["gate"])
    assert counts[-1] < 0.1 * open0, (open0, counts)
    assert _answered(r) < 0.2 * answered0, (answered0, _answered(r))
    # the lights come back: the frozen cache is right again and the gate reopens
    ds.lights.copy_(lights0)
    torch.cuda.synchronize()
    for _ in range(30):   # the bright frames' evidence decays by 0.8 per frame
        r.frame(f, accumulate=False)
        f += 1
    r.stream.synchronize()
    assert m.state()["gate"] > 0.5 * open0, (open0, m.state()["gate"])
    m.close()


def test_bad_policy_settings_are_rejected(terrain):
    from tfg_b200 import TfgError
    s, ds = terrain
    m = _mlp(s)
    for kw in ({"footprint": -0.01}, {"footprint": float("nan")}, {"train_fraction": -0.1},
               {"train_fraction": 1.5}, {"gate_threshold": -1.0}):
        r = NrcRenderer(ds, m, PARAMS, train_steps=1, max_records=4096, min_records=64, use_graph=False, **kw)
        with pytest.raises(TfgError):
            r.frame(1, accumulate=False)
    # the limits themselves are accepted
    for kw in ({"footprint": 0.0}, {"train_fraction": 0.0}, {"train_fraction": 1.0}):
        r = NrcRenderer(ds, m, PARAMS, train_steps=1, max_records=4096, min_records=64, use_graph=False, **kw)
        r.frame(1, accumulate=False)
        r.stream.synchronize()
        assert np.isfinite(r.image().cpu().numpy()).all()
    m.close()
