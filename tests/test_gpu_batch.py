"""Batched multi-scene cache frames (tfgNrcFrameBatch): several independent
scenes, each with its own cache model, advanced by one call as concurrent
branches, eagerly or as one replayed CUDA graph.  A frame of a scene in the
batch must equal the same frame rendered alone through tfgNrcFrame."""
import numpy as np
import pytest
import torch

from tfg_b200 import _lib
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
from tfg_b200.nrc import ColorMLP, NrcBatch, NrcRenderer

pytestmark = pytest.mark.gpu

PARAMS = pt.RenderParams(max_depth=6, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)
# (triangles, width, height, lights): more scenes than branches, mixed sizes
SPECS = [(6000, 96, 64, 1), (20000, 160, 96, 2), (3000, 64, 48, 3), (12000, 128, 80, 4), (8000, 80, 64, 2)]


@pytest.fixture(scope="module")
def batch_scenes(built):
    out = []
    for k, (tris, w, h, nl) in enumerate(SPECS):
        s = scenes.sized_terrain_scene(tris, w, h, nl, seed=300 + k)
        out.append((s, pt.DeviceScene(s, "cuda")))
    yield out
    for _, ds in out:
        ds.close()


# Scenes with different render settings cannot share a wavefront: the batch
# then renders each scene on its own branch.
MIXED = [PARAMS, pt.RenderParams(max_depth=5, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)]


def _renderers(batch_scenes, seed=11, graph=False, train_steps=2, mixed=False):
    rs = []
    for k, (s, ds) in enumerate(batch_scenes):
        m = ColorMLP(batch=16384, seed=seed + k)
        m.set_bounds(*s.bounds)
        prm = MIXED[k % 2] if mixed else PARAMS
        rs.append(NrcRenderer(ds, m, prm, train_steps=train_steps, max_records=4096, min_records=256,
                              use_graph=graph))
    return rs


def _close(rs):
    for r in rs:
        r.mlp.close()


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("graph", [False, True])
def test_batch_frame_equals_single_scene_frames(batch_scenes, graph, mixed):
    # With no training steps the cache model stays fixed and a frame is a
    # function of the scene, the model and the frame number (the training
    # record ring is filled through atomics, so trained models are not
    # bit-reproducible).  Both frames query the cache; with the graph, frame 6
    # captures and frame 7 replays the capture.
    single = _renderers(batch_scenes, train_steps=0, mixed=mixed)
    for r in single:
        r.frame(6, warmup=False, accumulate=False)
        r.frame(7, warmup=False, accumulate=False)
        r.stream.synchronize()
    want = [r.image().cpu().numpy().copy() for r in single]
    _close(single)
    rs = _renderers(batch_scenes, train_steps=0, mixed=mixed)
    b = NrcBatch(rs, use_graph=graph)
    b.frame(6, warmup=False)
    b.frame(7, warmup=False)
    b.stream.synchronize()
    for r, w in zip(rs, want):
        got = r.image().cpu().numpy()
        assert np.isfinite(got).all()
        np.testing.assert_array_equal(got, w)
    _close(rs)


def test_batched_frames_train_every_cache(batch_scenes):
    rs = _renderers(batch_scenes)
    b = NrcBatch(rs, use_graph=True)
    for f in range(6):
        b.frame(f, warmup=True)
    for f in range(6, 12):
        b.frame(f, warmup=False, accumulate=True)
    b.stream.synchronize()
    for r in rs:
        st = r.mlp.state()
        # 12 frames x 2 Adam steps once the ring holds enough records
        assert 12 <= st["adam_t"] <= 24
        assert np.isfinite(st["loss_ema"])
        img = r.mean_image().cpu().numpy()
        assert np.isfinite(img).all() and img.mean() > 0.0
    _close(rs)


def test_batch_rejects_shared_buffers(batch_scenes):
    rs = _renderers(batch_scenes[:2])
    rs[1].bufs = rs[0].bufs
    b = NrcBatch(rs, use_graph=False)
    with pytest.raises(_lib.TfgError):
        b.frame(0, warmup=True)
    _close(rs)


def test_empty_batch_is_a_no_op(built):
    assert _lib.lib.tfgNrcFrameBatch(0, None, 0, 0, None) == 0
    torch.cuda.synchronize()
