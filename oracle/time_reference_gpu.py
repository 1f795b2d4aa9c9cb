"""Time the reference's own GPU render kernel beside this project's drop-in
replacement -- TEST / MEASUREMENT INFRASTRUCTURE, not part of the product.

The reference's kernelRender_tiny (RenderKernel.cu, compiled unmodified for
sm_100a into oracle/_ref/libtfgref.so by build_oracle.py; 16x16 blocks as in
main.cpp) and tfgLaunchKernelRenderTiny run the same call -- scene, CWBVH,
camera, reference settings (depth 20, roulette after depth 10, the mesh does
not occlude shadow rays, transform triangle test) and RNG streams, so they
produce the same image -- on the 1920x1080 spheres-over-terrain scene
(1,000,480 triangles).  Prints one JSON line.  Needs a GPU:

    python oracle/time_reference_gpu.py [--frames N]
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import torch

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from oracle import oracle as orc            # noqa: E402
from tfg_b200 import pathtracer as pt       # noqa: E402
from tfg_b200 import scenes                 # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=10)
    args = ap.parse_args()
    ref = orc.ref()
    assert ref is not None and torch.cuda.is_available(), "needs a GPU and oracle/_ref/libtfgref.so"
    W, H = 1920, 1080
    scene = scenes.spheres_terrain(W, H)
    ds = pt.DeviceScene(scene, "cuda")
    img_ref = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    img_ours = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    # The reference kernel runs whole 16 x 16 blocks (68 block rows for 1080)
    # and writes the throughput of every thread without a bounds check, so the
    # per-pixel buffers get 16 spare rows.
    nb = pt.NrcBuffers(W * H + 16 * W, "cuda")

    def run_ref(frame):
        assert ref.ref_render_tiny(ds.camera.data_ptr(), None, 0, ds.lights.data_ptr(), ds.n_lights, W, H, frame,
                                   ds.bvh.ref.d_nodos, ds.bvh.ref.d_tris, ds.bvh.ref.num_nodos, ds.bvh.ref.num_tris,
                                   ds.bvh.d_primitivas, ds.n_mesh, img_ref.data_ptr(), nb.regs.data_ptr(),
                                   nb.counter.data_ptr(), nb.cap, nb.infer.data_ptr(), nb.thr.data_ptr(), 0, 0) == 0

    def run_ours(frame):
        pt.render_reference_call(ds, frame, img_ours, nrc=nb, stream=torch.cuda.default_stream())

    out = {}
    for name, fn in (("reference_kernel", run_ref), ("drop_in", run_ours)):
        for f in range(3):
            fn(f)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        for f in range(args.frames):
            fn(100 + f)
        e1.record(torch.cuda.default_stream())
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.frames
        out[name] = {"ms_per_frame_1spp": round(ms, 3), "mpaths_per_s": round(W * H / (ms * 1e-3) / 1e6, 1)}
    # primary-ray traversal: traverse_cwbvh (RenderKernel.cu build) against tfgTraceRays, same rays and BVH
    n = W * H
    rays = torch.zeros(n * 8, dtype=torch.float32, device="cuda")
    pt.camera_rays(ds, 0, rays)
    hits_r = torch.zeros(n * 4, dtype=torch.float32, device="cuda")
    hits_o = torch.zeros(n * 4, dtype=torch.float32, device="cuda")
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    tr = {"reference_traverse_cwbvh": lambda: ref.ref_trace(ds.bvh.ref.d_nodos, ds.bvh.ref.d_tris, rays.data_ptr(), n,
                                                             hits_r.data_ptr(), steps.data_ptr()),
          "tfgTraceRays": lambda: pt.trace_rays(ds, rays, hits_o, pt.TRIS_REF, stream=torch.cuda.default_stream())}
    for name, fn in tr.items():
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        for _ in range(args.frames):
            fn()
        e1.record(torch.cuda.default_stream())
        e1.synchronize()
        out[name] = {"grays_per_s": round(n * args.frames / (e0.elapsed_time(e1) * 1e-3) / 1e9, 3)}
    ids_r, ids_o = hits_r.view(-1, 4)[:, 3].cpu(), hits_o.view(-1, 4)[:, 3].cpu()
    out["primary_hit_ids_equal"] = bool(torch.equal(ids_r.view(torch.int32), ids_o.view(torch.int32)))
    # same RNG streams: the last frames rendered by both are frame 100 + frames - 1
    a, b = img_ref.cpu().double(), img_ours.cpu().double()
    out["image_relmse_between_them"] = float(((a - b) ** 2 / (a ** 2 + 1e-2)).mean())
    out["speedup"] = round(out["reference_kernel"]["ms_per_frame_1spp"] / out["drop_in"]["ms_per_frame_1spp"], 2)
    out["workload"] = ("1920x1080, 1 spp, spheres over terrain (1,000,480 tris), 2 point lights; reference settings: "
                       "depth 20, roulette after 10, mesh not occluding shadow rays, transform triangle test")
    print(json.dumps(out))
    ds.close()


if __name__ == "__main__":
    main()
