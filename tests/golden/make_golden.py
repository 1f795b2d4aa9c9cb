"""Generate the golden fixtures in this directory from the reference's own
GPU kernels (RenderKernel.cu / NrcKernel.cu compiled unmodified into
oracle/_ref/libtfgref.so by oracle/build_oracle.py).

Run on a machine with a CUDA GPU, from the repository root:

    python tests/golden/make_golden.py

The reference ships no tests, fixtures or golden vectors, so these outputs of
its kernels on small seeded inputs are what pins the CPU oracle without a
GPU (tests/test_golden_cpu.py).  Scenes and CWBVHs come from this project's
seeded generators and host builder; each fixture records a SHA-256 of the
BVH it was made on, so a changed builder is caught instead of compared.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as orc                     # noqa: E402
from tfg_b200 import bvh as hbvh                     # noqa: E402
from tfg_b200 import pathtracer as pt                # noqa: E402
from tfg_b200 import scenes                          # noqa: E402
from tfg_b200.structs import BOUNDS, CAMARA, COLOR, DATOS_MLP, REGISTRO   # noqa: E402

OUT = Path(__file__).resolve().parent

# (fixture name, scene factory) -- sizes are multiples of 16: the reference
# render kernel has no bounds guard.
RENDER_SCENES = {
    "reference_room": lambda: scenes.reference_room(32, 32, subdiv=2),
    "tiny_box": lambda: scenes.tiny_box(32, 32, subdiv=2),
}
RENDER_FRAMES = (1, 2)


def bvh_hash(hb) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(hb.nodes).tobytes())
    h.update(np.ascontiguousarray(hb.tris_ref).tobytes())
    return h.hexdigest()


def trace_rays_input(scene) -> np.ndarray:
    """Camera rays of frame 3 (oracle camera) plus 2048 seeded rays from inside the box."""
    cam = orc.camera_rays(scene.camera, scene.width, scene.height, 3)
    rng = np.random.default_rng(0)
    n = 2048
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = rng.uniform([-2.5, -1.9, -3.9], [2.5, 2.3, 5.4], (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 3] = 1e9
    return np.concatenate([cam.reshape(-1, 8), r]).astype(np.float32)


def kernel_inputs():
    """Seeded inputs of the element-wise NRC kernels (same generators as the
    GPU kernel tests)."""
    from tests.test_gpu_small_kernels import _bounds, _datos, _rand_colors, _regs
    rng = np.random.default_rng(11)
    W, H = 16, 16
    comp = [_rand_colors(rng, W * H, special=False) for _ in range(3)]
    n = 300
    regs = _regs(rng, n)
    tail = _rand_colors(rng, n, special=False)
    nd, batch = 700, 512
    datos = _datos(rng, nd)
    net = _rand_colors(rng, nd).reshape(-1)
    return dict(W=W, H=H, img=comp[0], pred=comp[1], thr=comp[2], regs=regs, tail=tail, nd=nd, batch=batch,
                datos=datos, net=net, bounds=_bounds())


def main() -> None:
    ref = orc.ref()
    assert ref is not None and torch.cuda.is_available(), "needs a GPU and oracle/_ref/libtfgref.so"
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()   # noqa: E731

    for name, make in RENDER_SCENES.items():
        s = make()
        ds = pt.DeviceScene(s, "cuda")
        hb = hbvh.build_host(hbvh.triangle_vertices(s.mesh))
        W, H = s.width, s.height
        imgs = []
        for f in RENDER_FRAMES:
            img = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
            nb = pt.NrcBuffers(W * H, "cuda")
            assert ref.ref_render_tiny(ds.camera.data_ptr(), ds.prims.data_ptr() if ds.prims is not None else None,
                                       ds.n_prims, ds.lights.data_ptr(), ds.n_lights, W, H, f, ds.bvh.ref.d_nodos,
                                       ds.bvh.ref.d_tris, ds.bvh.ref.num_nodos, ds.bvh.ref.num_tris,
                                       ds.bvh.d_primitivas, ds.n_mesh, img.data_ptr(), nb.regs.data_ptr(),
                                       nb.counter.data_ptr(), nb.cap, nb.infer.data_ptr(), nb.thr.data_ptr(), 0,
                                       0) == 0
            torch.cuda.synchronize()
            imgs.append(img.view(H, W, 3).cpu().numpy())
        np.savez_compressed(OUT / f"render_{name}.npz", frames=np.array(RENDER_FRAMES), images=np.stack(imgs),
                            bvh_sha256=bvh_hash(hb))
        ds.close()

    s = scenes.box_icosphere(64, 48, subdiv=3)
    ds = pt.DeviceScene(s, "cuda")
    hb = hbvh.build_host(hbvh.triangle_vertices(s.mesh))
    rays = trace_rays_input(s)
    n = len(rays)
    # every device buffer stays bound to a name until the kernels have run: a
    # temporary's memory goes back to torch's allocator at once
    drays = torch.from_numpy(rays.reshape(-1).copy()).cuda()
    hits = torch.zeros(n * 4, dtype=torch.float32, device="cuda")
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert ref.ref_trace(ds.bvh.ref.d_nodos, ds.bvh.ref.d_tris, drays.data_ptr(), n, hits.data_ptr(),
                         steps.data_ptr()) == 0
    torch.cuda.synchronize()
    np.savez_compressed(OUT / "trace_box_icosphere.npz", rays=rays, hits=hits.view(n, 4).cpu().numpy(),
                        steps=steps.cpu().numpy(), bvh_sha256=bvh_hash(hb))
    ds.close()

    k = kernel_inputs()
    W, H = k["W"], k["H"]
    img, dpred, dthr = dev(k["img"]), dev(k["pred"]), dev(k["thr"])
    assert ref.ref_composite(img.data_ptr(), dpred.data_ptr(), dthr.data_ptr(), W, H) == 0
    regs, dtail = dev(k["regs"]), dev(k["tail"])
    tail_out = torch.zeros(len(k["regs"]) * DATOS_MLP.itemsize, dtype=torch.uint8, device="cuda")
    targets = torch.zeros(len(k["regs"]) * DATOS_MLP.itemsize, dtype=torch.uint8, device="cuda")
    assert ref.ref_targets(regs.data_ptr(), dtail.data_ptr(), targets.data_ptr(), len(k["regs"])) == 0
    assert ref.ref_tail(regs.data_ptr(), tail_out.data_ptr(), len(k["regs"])) == 0
    nd, batch = k["nd"], k["batch"]
    idx = torch.zeros(batch, dtype=torch.int32, device="cuda")
    assert ref.ref_indices(idx.data_ptr(), nd, batch, 12345) == 0
    dd = dev(k["datos"])
    bb = k["bounds"].ctypes.data
    tin = torch.zeros(batch * 15, device="cuda")
    ttg = torch.zeros(batch * 3, device="cuda")
    assert ref.ref_train_rows(dd.data_ptr(), idx.data_ptr(), batch, 15, 3, bb, tin.data_ptr(), ttg.data_ptr()) == 0
    irows = torch.zeros(nd * 15, device="cuda")
    assert ref.ref_infer_rows(dd.data_ptr(), nd, 15, irows.data_ptr(), bb) == 0
    scrub = dev(np.zeros(nd, COLOR))
    dnet = torch.from_numpy(k["net"].copy()).cuda()
    assert ref.ref_scrub(dnet.data_ptr(), scrub.data_ptr(), nd) == 0
    cams = {}
    for (cw, ch) in ((512, 512), (1920, 1080), (7, 3)):
        c = torch.zeros(CAMARA.itemsize, dtype=torch.uint8, device="cuda")
        assert ref.ref_camera(c.data_ptr(), cw, ch) == 0
        cams[f"camera_{cw}x{ch}"] = c
    torch.cuda.synchronize()
    host = lambda t: t.cpu().numpy()   # noqa: E731
    np.savez_compressed(
        OUT / "nrc_kernels.npz",
        comp_img=k["img"], comp_pred=k["pred"], comp_thr=k["thr"], comp_out=host(img).view(np.float32).reshape(-1, 3),
        regs=k["regs"].view(np.uint8), tail=k["tail"], targets=host(targets), tail_out=host(tail_out),
        nd=nd, batch=batch, datos=k["datos"].view(np.uint8), bounds=k["bounds"].view(np.uint8),
        indices=host(idx), train_in=host(tin), train_tgt=host(ttg), infer_rows=host(irows), net=k["net"],
        scrub=host(scrub), **{key: host(v) for key, v in cams.items()})
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
