"""The reference-side binding on the GPU: the reference's own call shapes,
compiled against its unmodified headers (tfg_b200/dropin/libtfgdropin.so),
give exactly what the C ABI gives when called directly.

* launchKernelRenderTiny(dim3, dim3, ..., TinyBVHD_GPU, ..., ImagenGPU, ...)
  (RenderKernel.h:55-61) renders the image tfgLaunchKernelRenderTiny renders,
  bit for bit;
* class TinyBVH (tinybvh_wrapper.h:22-50) builds the tree tfgTinyBVHConstruir
  builds, and rendering through it gives the same image;
* class ColorMLP (mlp.h:19-44) trains and answers as tfgMlpCreate /
  tfgMlpTrainStep / tfgMlpInference do (to the order of the FP32 gradient
  sums, which atomics leave open)."""
import ctypes
from ctypes import c_float, c_int, c_uint, c_void_p

import numpy as np
import pytest
import torch

from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
from tfg_b200.dropin import build_dropin
from tfg_b200.nrc import ColorMLP
from tfg_b200.structs import DATOS_MLP

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin(built):
    path = build_dropin.build()
    if path is None:
        pytest.skip("reference-side binding not built (needs the reference's headers)")
    lib = ctypes.CDLL(str(path))
    lib.dropin_render_tiny.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_int, c_void_p,
                                       c_void_p, c_uint, c_uint, c_void_p, c_int, c_void_p, c_void_p]
    lib.dropin_bvh_build.restype = c_void_p
    lib.dropin_bvh_build.argtypes = [c_void_p, c_int, ctypes.POINTER(c_uint), ctypes.POINTER(c_uint),
                                     ctypes.POINTER(c_uint)]
    lib.dropin_bvh_render.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_int,
                                      c_void_p, c_void_p]
    lib.dropin_bvh_free.argtypes = [c_void_p]
    lib.dropin_mlp_train_infer.restype = c_float
    lib.dropin_mlp_train_infer.argtypes = [c_void_p, c_uint, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_uint]
    return lib


@pytest.fixture(scope="module")
def room(built):
    s = scenes.reference_room(96, 64, subdiv=3)
    ds = pt.DeviceScene(s, "cuda")
    yield s, ds
    ds.close()


def _abi_image(ds, frame):
    W, H = ds.scene.width, ds.scene.height
    img = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    pt.render_reference_call(ds, frame, img)
    torch.cuda.synchronize()
    return img.cpu().numpy()


def test_reference_call_shape_renders_the_c_abi_image(dropin, room):
    s, ds = room
    W, H = s.width, s.height
    for frame in (0, 7):
        img = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
        thr = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")   # main.cpp:908-930 always passes one
        assert dropin.dropin_render_tiny(ds.camera.data_ptr(), ds.prims.data_ptr(), ds.n_prims,
                                         ds.lights.data_ptr(), ds.n_lights, W, H, frame, ds.bvh.ref.d_nodos,
                                         ds.bvh.ref.d_tris, ds.bvh.ref.num_nodos, ds.bvh.ref.num_tris,
                                         ds.bvh.d_primitivas, ds.n_mesh, img.data_ptr(), thr.data_ptr()) == 0
        got = img.cpu().numpy()
        want = _abi_image(ds, frame)
        assert np.isfinite(got).all() and got.mean() > 0
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_tinybvh_class_builds_the_c_abi_tree(dropin, room):
    s, ds = room
    W, H = s.width, s.height
    nn, nt, npr = c_uint(), c_uint(), c_uint()
    mesh = np.ascontiguousarray(s.mesh)
    h = dropin.dropin_bvh_build(mesh.ctypes.data, len(mesh), ctypes.byref(nn), ctypes.byref(nt), ctypes.byref(npr))
    try:
        assert (nn.value, nt.value, npr.value) == (ds.bvh.ref.num_nodos, ds.bvh.ref.num_tris, ds.n_mesh)
        img = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
        thr = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
        assert dropin.dropin_bvh_render(h, ds.camera.data_ptr(), ds.prims.data_ptr(), ds.n_prims,
                                        ds.lights.data_ptr(), ds.n_lights, W, H, 3, img.data_ptr(),
                                        thr.data_ptr()) == 0
        got = img.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), _abi_image(ds, 3).view(np.uint32))
    finally:
        dropin.dropin_bvh_free(h)


def test_colormlp_class_trains_and_answers_as_the_c_abi(dropin):
    lo, hi = (-6.0, -4.0, -10.0), (6.0, 6.0, 2.0)
    rng = np.random.default_rng(4)
    n_avail, n = 30000, 5000
    d = np.zeros(n_avail, DATOS_MLP)
    for j, k in enumerate("xyz"):
        d["posicion"][k] = rng.uniform(lo[j], hi[j], n_avail)
        d["direccion"][k] = rng.uniform(0, 1, n_avail)
        d["normal"][k] = rng.uniform(0, 1, n_avail)
    for k in "rgb":
        d["difuso"][k] = rng.uniform(0, 1, n_avail)
        d["color"][k] = rng.uniform(0, 2, n_avail)
    dd = torch.from_numpy(d.view(np.uint8).copy()).cuda()
    q = torch.from_numpy(d[:n].view(np.uint8).copy()).cuda()
    out_a = torch.zeros(n * 3, device="cuda")
    lo_a, hi_a = np.array(lo), np.array(hi)
    loss_a = dropin.dropin_mlp_train_infer(dd.data_ptr(), n_avail, 3, lo_a.ctypes.data, hi_a.ctypes.data,
                                           q.data_ptr(), out_a.data_ptr(), n)
    m = ColorMLP(batch=16384, seed=1337)        # the class's seed
    m.set_bounds(lo, hi)
    loss_b = 0.0
    for _ in range(3):
        loss_b = m.train_step(dd, n_avail)
    out_b = torch.zeros(n * 3, device="cuda")
    m.inference(q, out_b, n)
    torch.cuda.synchronize()
    m.close()
    assert loss_a > 0 and abs(loss_a - loss_b) <= 1e-5 * loss_b, (loss_a, loss_b)
    a, b = out_a.cpu().numpy(), out_b.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-3 * (np.abs(b).mean() + 1e-3), float(np.abs(a - b).max())
