"""The allocation-free render entry point (tfgRenderPassStatic).

Some callers cannot allocate device memory: code that runs while another
thread captures a CUDA graph in global mode, engines that hand the library a
fixed memory budget, real-time threads that must not wait on the allocator.
tfgRenderPassStatic renders from a fixed static scratch array instead of the
library's allocated workspace.  Called through the C ABI, twice in a row, it
must produce what the allocating entry point (tfgRenderPass) produces for the
same inputs, to the render tests' tolerance (relMSE <= 1e-4), and it must
refuse images larger than its scratch with a clear error.  This file is
collected last so that a run stopping at the first failure has run every
other test first."""
import numpy as np
import pytest
import torch

from tests.helpers import rel_mse
from tfg_b200 import _lib
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene_ds(built):
    s = scenes.box_icosphere(96, 64, subdiv=3)
    ds = pt.DeviceScene(s, "cuda")
    yield s, ds
    ds.close()


@pytest.mark.parametrize("fmt", [pt.TRIS_WATERTIGHT, pt.TRIS_REF])
def test_static_scratch_matches_allocating_entry(scene_ds, fmt):
    s, ds = scene_ds
    W, H = s.width, s.height
    params = pt.RenderParams(max_depth=8, rr_min_depth=3, shadow_mesh=1, tri_format=fmt)
    frames = (11, 12)
    want = []
    for f in frames:
        img = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
        pt.render_pass(ds, params, f, img)
        torch.cuda.synchronize()
        want.append(img.view(H, W, 3).cpu().numpy())
    # two calls in a row of the allocation-free entry point
    got = []
    for f in frames:
        img = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
        pt.render_pass_static(ds, params, f, img)
        torch.cuda.synchronize()
        got.append(img.view(H, W, 3).cpu().numpy())
    for g, w in zip(got, want):
        assert np.isfinite(g).all()
        assert g.mean() > 0.0
        assert rel_mse(g, w) <= 1e-4


def test_static_scratch_accumulates(scene_ds):
    s, ds = scene_ds
    W, H = s.width, s.height
    params = pt.RenderParams(max_depth=5, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT, spp=3,
                             accumulate=1)
    a = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    b = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    pt.render_pass(ds, params, 40, None, a)
    pt.render_pass_static(ds, params, 40, None, b)
    torch.cuda.synchronize()
    assert rel_mse(b.cpu().numpy() / 3, a.cpu().numpy() / 3) <= 1e-4


def test_static_scratch_rejects_oversize_images(built):
    s = scenes.box_icosphere(160, 128, subdiv=1)   # 20480 pixels > 16384
    ds = pt.DeviceScene(s, "cuda")
    with pytest.raises(_lib.TfgError) as e:
        pt.render_pass_static(ds, pt.RenderParams(), 0, torch.zeros(160 * 128 * 3, device="cuda"))
    assert e.value.code == 10001 and "16384" in str(e.value)
    ds.close()
