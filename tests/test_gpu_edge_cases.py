"""Edge cases of the render entry points against the CPU oracle: ragged image
sizes (not multiples of the reference's 16x16 blocks), the deepest allowed
paths, scenes without lights, without a mesh or without analytic primitives,
and the limits the entry points must reject."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from tests.helpers import oracle_image, reference_params, rel_mse
from tfg_b200 import TfgError
from tfg_b200 import bvh as hbvh
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
from tfg_b200.scenes import Scene

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _mine(ds, params, frame):
    W, H = ds.scene.width, ds.scene.height
    img = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    pt.render_pass(ds, params, frame, img)
    torch.cuda.synchronize()
    return img.view(H, W, 3).cpu().numpy()


def _compare(s, max_depth=5, rr=3, frames=4):
    ds = pt.DeviceScene(s, "cuda")
    params = pt.RenderParams(max_depth=max_depth, rr_min_depth=rr, shadow_mesh=1, tri_format=pt.TRIS_REF)
    prm = reference_params(max_depth=max_depth, rr_min_depth=rr, shadow_mesh=1)
    hb = hbvh.build_host(hbvh.triangle_vertices(s.mesh)) if len(s.mesh) else None
    mine = np.zeros((s.height, s.width, 3))
    cpu = np.zeros_like(mine)
    for f in range(frames):
        mine += _mine(ds, params, 40 + f)
        if hb is not None:
            cpu += oracle_image(orc, s, hb, 40 + f, prm)
    ds.close()
    return mine / frames, (cpu / frames if hb is not None else None)


@pytest.mark.parametrize("wh", [(37, 23), (1, 1), (129, 3)])
def test_ragged_image_sizes(built, wh):
    W, H = wh
    s = scenes.box_icosphere(W, H, subdiv=3)
    mine, cpu = _compare(s)
    assert np.isfinite(mine).all()
    assert rel_mse(mine, cpu) <= TOL


def test_deepest_paths(built):
    # a closed box: paths survive to the 64-bounce limit often enough to matter
    s = scenes.box_icosphere(48, 32, subdiv=2)
    mine, cpu = _compare(s, max_depth=64, rr=60, frames=2)
    assert rel_mse(mine, cpu) <= TOL


def test_scene_without_lights_is_black(built):
    base = scenes.box_icosphere(32, 32, subdiv=2)
    s = Scene(base.prims, base.mesh, base.lights[:0], base.camera, 32, 32, bounds=base.bounds)
    mine, cpu = _compare(s, frames=1)
    assert np.abs(mine).max() == 0.0 and np.abs(cpu).max() == 0.0


def test_scene_without_analytic_primitives(built):
    base = scenes.box_icosphere(40, 24, subdiv=3)
    s = Scene(base.prims[:0], base.mesh, base.lights, base.camera, 40, 24, bounds=base.bounds)
    mine, cpu = _compare(s)
    assert rel_mse(mine, cpu) <= TOL


def test_scene_without_mesh_renders_the_analytic_primitives(built):
    base = scenes.reference_room(48, 32, subdiv=2)
    s = Scene(base.prims, base.mesh[:0], base.lights, base.camera, 48, 32, bounds=base.bounds)
    mine, _ = _compare(s, frames=2)
    assert np.isfinite(mine).all() and mine.max() > 0.0


def test_limits_are_rejected(built):
    s = scenes.box_icosphere(16, 16, subdiv=1)
    ds = pt.DeviceScene(s, "cuda")
    img = torch.zeros(16 * 16 * 3, device="cuda")
    for bad in (pt.RenderParams(max_depth=65), pt.RenderParams(max_depth=0), pt.RenderParams(spp=0),
                pt.RenderParams(tri_format=7)):
        with pytest.raises(TfgError):
            pt.render_pass(ds, bad, 0, img)
    ds.close()
