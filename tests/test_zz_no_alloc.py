"""The allocation-free render entry point (tfgRenderPassStatic).

Some callers cannot allocate device memory: code that runs while another
thread captures a CUDA graph in global mode (cudaMalloc is not allowed then),
engines that hand the library a fixed memory budget, real-time threads that
must not wait on the allocator.  tfgRenderPassStatic renders from a fixed
static scratch array instead of the library's allocated workspace.

Called through the C ABI, twice in a row, it must produce exactly what the
allocating entry point (tfgRenderPass) produces for the same inputs (a launch
setting never changes what a path computes, so the images are equal bit for
bit), leave the device's free memory unchanged once warm, work as the first
render call of a fresh process, and refuse images larger than its scratch with
a clear error.  This file is collected last so that a run stopping at the
first failure has run every other test first."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from tfg_b200 import _lib
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def scene_ds(built):
    s = scenes.box_icosphere(96, 64, subdiv=3)
    ds = pt.DeviceScene(s, "cuda")
    yield s, ds
    ds.close()


def _image(render, ds, params, frame):
    W, H = ds.scene.width, ds.scene.height
    img = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    render(ds, params, frame, img)
    torch.cuda.synchronize()
    return img.view(H, W, 3).cpu().numpy()


@pytest.mark.parametrize("fmt", [pt.TRIS_WATERTIGHT, pt.TRIS_REF])
def test_static_scratch_matches_allocating_entry(scene_ds, fmt):
    _, ds = scene_ds
    params = pt.RenderParams(max_depth=8, rr_min_depth=3, shadow_mesh=1, tri_format=fmt)
    frames = (11, 12)
    want = [_image(pt.render_pass, ds, params, f) for f in frames]
    # two calls in a row of the allocation-free entry point
    got = [_image(pt.render_pass_static, ds, params, f) for f in frames]
    for g, w in zip(got, want):
        assert np.isfinite(g).all()
        assert g.mean() > 0.0
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))
    assert not np.array_equal(got[0], got[1])   # the frame number reaches the RNG seeds


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
    assert torch.equal(a, b)


def test_static_scratch_rejects_oversize_images(built):
    s = scenes.box_icosphere(160, 128, subdiv=1)   # 20480 pixels > 16384
    ds = pt.DeviceScene(s, "cuda")
    with pytest.raises(_lib.TfgError) as e:
        pt.render_pass_static(ds, pt.RenderParams(), 0, torch.zeros(160 * 128 * 3, device="cuda"))
    assert e.value.code == 10001 and "16384" in str(e.value)
    ds.close()


# Run in a child process: the static entry point is the first render call the
# process makes (no tfgRenderPass before it has set up a workspace), a warm
# second call must leave cudaMemGetInfo's free bytes unchanged, and both calls
# must equal the allocating entry point afterwards.
_FRESH = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
s = scenes.box_icosphere(128, 96, subdiv=3)
ds = pt.DeviceScene(s, "cuda")
n = s.width * s.height * 3
params = pt.RenderParams(max_depth=8, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)
imgs = [torch.zeros(n, dtype=torch.float32, device="cuda") for _ in range(3)]
torch.cuda.synchronize()
pt.render_pass_static(ds, params, 5, imgs[0])
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
pt.render_pass_static(ds, params, 6, imgs[1])
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
assert free1 == free0, f"free device memory changed across a warm static call: {free0} -> {free1}"
for k, f in enumerate((5, 6)):
    pt.render_pass(ds, params, f, imgs[2])
    torch.cuda.synchronize()
    assert torch.equal(imgs[k], imgs[2]), f"frame {f}: static and allocating passes differ"
assert float(imgs[0].mean()) > 0.0
ds.close()
print("fresh-process static pass ok")
"""


def test_static_first_call_of_a_fresh_process_allocates_nothing(built):
    env = dict(os.environ)
    res = subprocess.run([sys.executable, "-c", _FRESH, str(ROOT)], capture_output=True, text=True, timeout=600,
                         env=env)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-4000:]
    assert "fresh-process static pass ok" in res.stdout
