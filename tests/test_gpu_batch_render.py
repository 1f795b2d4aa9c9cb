"""Several scenes in one wavefront series (tfgRenderPassBatch and the
batched cache frame): every stage is one launch for all scenes, and each
scene's image must equal what a single-scene pass gives for it, bit for bit
-- scenes of different sizes, light counts, with and without analytic
primitives or a mesh, under any launch tuning."""
import numpy as np
import pytest
import torch

from tfg_b200 import TfgError
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
from tfg_b200.scenes import Scene

pytestmark = pytest.mark.gpu

PARAMS = pt.RenderParams(max_depth=6, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)


def _scene_set():
    out = [scenes.sized_terrain_scene(tris, w, h, nl, seed=700 + k)
           for k, (tris, w, h, nl) in enumerate([(6000, 96, 64, 1), (20000, 160, 96, 3), (3000, 37, 23, 4)])]
    room = scenes.reference_room(48, 40, subdiv=2)         # analytic spheres / planes + mesh
    out.append(room)
    out.append(Scene(room.prims, room.mesh[:0], room.lights, room.camera, 48, 40, bounds=room.bounds))  # no mesh
    out.append(scenes.box_icosphere(64, 48, subdiv=3))
    return out


@pytest.fixture(scope="module")
def dss(built):
    ds = [pt.DeviceScene(s, "cuda") for s in _scene_set()]
    yield ds
    for d in ds:
        d.close()


@pytest.fixture(autouse=True)
def default_tuning():
    pt.set_tuning(pt.RenderTuning.default())
    yield
    pt.set_tuning(pt.RenderTuning.default())


def _buffers(dss):
    imgs = [torch.zeros(d.scene.width * d.scene.height * 3, device="cuda") for d in dss]
    accs = [torch.zeros_like(i) for i in imgs]
    return imgs, accs


def _singles(dss, params, frame):
    imgs, accs = _buffers(dss)
    for d, i, a in zip(dss, imgs, accs):
        pt.render_pass(d, params, frame, i, a)
    torch.cuda.synchronize()
    return [x.cpu().numpy() for x in imgs], [x.cpu().numpy() for x in accs]


def _batch(dss, params, frame):
    imgs, accs = _buffers(dss)
    pt.render_pass_batch(dss, params, frame, imgs, accs)
    torch.cuda.synchronize()
    return [x.cpu().numpy() for x in imgs], [x.cpu().numpy() for x in accs]


@pytest.mark.parametrize("fmt", [pt.TRIS_WATERTIGHT, pt.TRIS_REF])
def test_batch_pass_equals_single_scene_passes(dss, fmt):
    p = pt.RenderParams(**{**PARAMS.__dict__, "tri_format": fmt, "spp": 3, "accumulate": 1})
    want_i, want_a = _singles(dss, p, 17)
    got_i, got_a = _batch(dss, p, 17)
    for k, (gi, ga, wi, wa) in enumerate(zip(got_i, got_a, want_i, want_a)):
        assert np.isfinite(ga).all()
        np.testing.assert_array_equal(gi, wi, err_msg=f"scene {k}")
        np.testing.assert_array_equal(ga, wa, err_msg=f"scene {k}")
    assert max(a.max() for a in got_a) > 0


def test_batch_pass_under_tuning(dss):
    p = pt.RenderParams(**{**PARAMS.__dict__, "spp": 4, "accumulate": 1})
    want_i, want_a = _singles(dss, p, 3)
    total = sum(d.scene.width * d.scene.height for d in dss)
    for t in (pt.RenderTuning(wavefront_paths=1024), pt.RenderTuning(wavefront_paths=total + 333),
              pt.RenderTuning(wavefront_paths=4 * total, trace_threads=64, refill_min=3),
              pt.RenderTuning(wavefront_paths=2 * total, overlap_shadow=1)):
        pt.set_tuning(t)
        got_i, got_a = _batch(dss, p, 3)
        for gi, ga, wi, wa in zip(got_i, got_a, want_i, want_a):
            np.testing.assert_array_equal(gi, wi, err_msg=str(t))
            np.testing.assert_array_equal(ga, wa, err_msg=str(t))


def test_more_than_sixteen_scenes(built):
    scs = [scenes.sized_terrain_scene(2000 + 300 * k, 24 + 4 * k, 16 + 2 * k, 1 + k % 4, seed=900 + k) for k in range(18)]
    ds = [pt.DeviceScene(s, "cuda") for s in scs]
    p = pt.RenderParams(**{**PARAMS.__dict__, "spp": 2, "accumulate": 1})
    want_i, want_a = _singles(ds, p, 5)
    got_i, got_a = _batch(ds, p, 5)
    for gi, ga, wi, wa in zip(got_i, got_a, want_i, want_a):
        np.testing.assert_array_equal(gi, wi)
        np.testing.assert_array_equal(ga, wa)
    for d in ds:
        d.close()


def test_batch_rejects_bad_scenes(dss):
    p = pt.RenderParams(**PARAMS.__dict__)
    with pytest.raises(TfgError):
        pt.render_pass_batch(dss, pt.RenderParams(max_depth=0), 0)
    bad = pt.DeviceScene(scenes.box_icosphere(16, 16, subdiv=1), "cuda")
    bad.scene = Scene(bad.scene.prims, bad.scene.mesh, bad.scene.lights, bad.scene.camera, 0, 16,
                      bounds=bad.scene.bounds)
    with pytest.raises(TfgError):
        pt.render_pass_batch([dss[0], bad], p, 0)
    bad.close()
