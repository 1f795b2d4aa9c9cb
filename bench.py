"""Benchmark: plain path tracing at 1920x1080 on the ~1.0M-triangle scene.

Workload (one step = one frame): 16 displaced icospheres (subdivision 5) on a
fractal heightfield, 1,000,480 triangles, two point lights, albedo
U[0.1, 0.9]; 1920x1080 pixels x 64 samples per pixel, max depth 8, Russian
roulette from depth 3, mesh-occluded shadow rays, watertight triangle test.
Seeded synthetic data.  Metric: Mpaths/s (paths = pixels x spp), ms/frame.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU runs are independent replicas (one process per GPU, launched by
torch.distributed.run); value = all ranks' paths / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

W_PX, H_PX, SPP, DEPTH, RR = 1920, 1080, 64, 8, 3
METRIC = "Mpaths/s & ms/frame @1080p"
WORKLOAD = "plain path tracing, 1920x1080, 64 spp, depth 8, RR from depth 3, 16 displaced icospheres + fractal terrain (1,000,480 tris), 2 point lights"


# DRAM bytes (read + write) per closest-hit ray, measured with ncu over the
# eight closest-hit launches of `bench.py --profile-pass --wavefront-samples K`
# (profiles/k_trace_k_shadow_dram_1080p.md, k_trace_l2_issue_1080p.md): 306.4 MB
# over 4,001,265 rays with one sample per wavefront, 4,041 MB over 64,020,240
# rays with 16; the cold first touch of the tree is shared by more rays in
# larger wavefronts.
TRACE_DRAM_BYTES_PER_RAY = {1: 76.57, 16: 63.12}


# ncu counters of the closest-hit kernel on the bench frame (one-sample pass,
# all eight bounces; profiles/k_trace_l2_issue_1080p.md): L2 bytes
# (lts__t_bytes.sum) per closest-hit ray traced, the share of issue slots
# used (sm__inst_issued.avg.per_cycle_active / 4) and the SIMT efficiency
# (smsp__thread_inst_executed_per_inst_executed.ratio / 32), over the pass's
# 4,001,265 rays, weighted by duration and by instructions respectively.
TRACE_L2_BYTES_PER_RAY = 508.0
TRACE_ISSUE_FRAC = 0.561
TRACE_SIMT_EFFICIENCY = 0.406
# k_shadow's active lanes per instruction (of 32) on the first bounce of the
# one-sample pass (profiles/k_trace_k_shadow_bounce0_full_1080p.md: 15.18).
SHADOW_SIMT_EFFICIENCY = 0.474


def l2_gather_peak(dev) -> dict:
    """Random-gather bandwidth of L2 (tfgL2GatherPass): 80-byte records at
    hashed indices of a 64 MiB table (L2-resident, as the benchmark scene's
    CWBVH is), 1184 x 256 threads x 256 reads per pass, best of 10 passes
    timed with CUDA events after 3 warm-ups."""
    import torch

    from tfg_b200 import _lib
    records = (64 << 20) // 80
    table = torch.randint(0, 1 << 30, (records * 20,), dtype=torch.int32, device=dev)
    sink = torch.zeros(1, dtype=torch.int32, device=dev)
    blocks, reads = 148 * 8, 256
    stream = torch.cuda.current_stream()

    def one(seed):
        _lib.call("tfgL2GatherPass", table.data_ptr(), records, reads, seed, sink.data_ptr(), blocks,
                  stream.cuda_stream)

    for k in range(3):
        one(k)
    torch.cuda.synchronize()
    best = float("inf")
    for k in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        one(100 + k)
        e1.record(stream)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    nbytes = 80.0 * blocks * 256 * reads
    del table
    return {"gbs": round(nbytes / (best * 1e-3) / 1e9, 1), "ms": round(best, 4), "bytes": int(nbytes),
            "how": "80 B records at hashed indices of a 64 MiB table, 1184 x 256 threads x 256 reads, best of 10"}


def trace_traffic(wavefront_paths: int, n_px: int, rays_per_launch: float) -> int:
    """DRAM bytes per closest-hit launch: the measured bytes per ray of the
    nearest captured wavefront size (1 or 16 samples) times the rays of an
    average launch."""
    k = max(1, wavefront_paths // n_px) if wavefront_paths else 1
    return int(round(TRACE_DRAM_BYTES_PER_RAY[1 if k < 4 else 16] * rays_per_launch))


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        # Start timing only once the sampler has written its first sample:
        # its start-up (driver initialisation) then falls outside the timed
        # region, and the region is sampled from its first 200 ms on.
        t_end = time.perf_counter() + 10.0
        while self.proc is not None and self.proc.poll() is None and time.perf_counter() < t_end:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """Largest value over the ranks (device times: the job is as slow as its
    slowest replica).  NCCL reduces a CUDA tensor, gloo a host one."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(paths_per_rank: int, ms_max: float, world: int) -> float:
    """Whole-job Mpaths/s of `world` replicas that each trace `paths_per_rank`
    paths, timed by the slowest rank."""
    return world * paths_per_rank / (ms_max * 1e-3) / 1e6


def replica_frame(rank: int, step: int, steps: int) -> int:
    """First frame number of timed step `step` on `rank`: every replica renders
    its own frames (rank r's steps are frames 1 + SPP * (r * steps + s) ..),
    so N ranks trace N distinct 64-spp frames per step; rank 0's are the
    single-GPU run's."""
    return 1 + SPP * (rank * steps + step)


def cpu_oracle_sample(scene, hb, rows: int, nthreads: int, frame: int = 1) -> tuple[float, int]:
    """Time the CPU oracle (a restatement of the reference path tracer) on a
    band of `rows` image rows at 1 spp; returns (seconds, paths)."""
    import ctypes

    import numpy as np

    from oracle import oracle as orc
    from tfg_b200.pathtracer import RenderParams
    prm = RenderParams(max_depth=DEPTH, rr_min_depth=RR, shadow_mesh=1).c()
    y0 = max(0, H_PX // 2 - rows // 2)
    img = np.zeros((rows, W_PX, 3), np.float32)
    t0 = time.perf_counter()
    orc.cpu.orc_render(orc.p(scene.prims), len(scene.prims), orc.p(scene.lights), len(scene.lights),
                       orc.p(hb.nodes), orc.p(hb.tris_ref), orc.p(scene.mesh), len(scene.mesh),
                       orc.p(scene.camera), W_PX, H_PX, frame, ctypes.addressof(prm), y0, y0 + rows, orc.p(img),
                       None, None, None, None, 0, 0, nthreads)
    return time.perf_counter() - t0, rows * W_PX


def reference_arm(args):
    """The reference's path tracer on the host cores: the reference ships no
    CPU renderer, so this is the CPU restatement (oracle), all threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from tfg_b200 import bvh as hbvh
    from tfg_b200 import scenes
    scene = scenes.spheres_terrain(W_PX, H_PX)
    hb = hbvh.build_host(hbvh.triangle_vertices(scene.mesh))
    nthreads = os.cpu_count() or 1
    rows = H_PX
    for _ in range(args.warmup):
        cpu_oracle_sample(scene, hb, 8, nthreads)
    secs, paths = 0.0, 0
    for s in range(args.steps):
        dt, n = cpu_oracle_sample(scene, hb, rows, nthreads, frame=1 + s)
        secs += dt
        paths += n
    v = paths / secs / 1e6
    sample = (f"each step: the full 1920x1080 frame at 1 spp (1/64 of a 64-spp frame), depth {DEPTH}, "
              f"RR from {RR}; warm-up steps: 8 rows")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "Mpaths/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * secs / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
        "data": "synthetic (seeded)", "config": {"workload": WORKLOAD, "sample": sample},
        "cpu_baseline": {"value": round(v, 4), "unit": "Mpaths/s", "cores": nthreads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(v, 4), "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def nrc_eval(scene, ds, dev, ref_spp: int = 4096, frames: int = 300) -> dict:
    """Online radiance caching at 1920x1080 (1 spp per frame, camera orbiting
    1 degree per frame, 4 x 16384 training samples per frame after the
    reference's 48 warm-up frames) against plain path tracing at equal GPU
    time.  Both are scored by relMSE against a `ref_spp` plain path-traced
    image of the final camera pose, accumulated in FP64 (64-sample FP32
    batches summed in FP64)."""
    import numpy as np
    import torch

    from tfg_b200 import pathtracer as pt
    from tfg_b200 import scenes as sc
    from tfg_b200.nrc import ColorMLP, NrcRenderer

    params = pt.RenderParams(max_depth=DEPTH, rr_min_depth=RR, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)
    # launch settings tuned for single-sample passes; cache frames and the
    # plain passes they are compared with both use them
    tuning_1spp, _ = pt.autotune(ds, params, repeats=3)
    mlp = ColorMLP(batch=16384, seed=2024)
    mlp.set_bounds(*scene.bounds)
    r = NrcRenderer(ds, mlp, params, train_steps=4, use_graph=True)

    def set_pose(k):
        cam = sc.orbit_camera((0.0, -1.0, -7.0), 13.0, 2.8, float(k), W_PX, H_PX)
        ds.camera.copy_(torch.from_numpy(cam.view("u1").copy()).to(dev), non_blocking=False)

    for f in range(48):
        with torch.cuda.stream(r.stream):
            set_pose(0)
        r.frame(f, warmup=True, accumulate=False)
    for k in range(frames):
        with torch.cuda.stream(r.stream):
            set_pose(k)
        r.frame(48 + k, accumulate=False)
    r.stream.synchronize()
    # time cache frames and plain passes at the final pose
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(r.stream)
    for k in range(10):
        r.frame(10_000 + k, accumulate=False)
    e1.record(r.stream)
    e1.synchronize()
    t_nrc = e0.elapsed_time(e1) / 10
    nrc_img = r.image().cpu().numpy().astype(np.float64)
    img = torch.zeros(W_PX * H_PX * 3, dtype=torch.float32, device=dev)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    for k in range(10):
        pt.render_pass(ds, params, 20_000 + k, img)
    p1.record()
    p1.synchronize()
    t_pt = p0.elapsed_time(p1) / 10
    spp_eq = max(1, int(round(t_nrc / t_pt)))
    plain = pt.accumulate_spp(ds, params, spp_eq, 30_000).cpu().numpy().astype(np.float64)
    ref = np.zeros_like(plain)
    for b in range(ref_spp // 64):
        ref += pt.accumulate_spp(ds, params, 64, 1_000_000 + 64 * b).cpu().numpy().astype(np.float64)
    ref /= ref_spp // 64

    def rel(x):
        return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))

    e_nrc, e_pt = rel(nrc_img), rel(plain)
    # plain path tracing is unbiased: relMSE x time is its equal-time figure of merit
    ratio_time = (e_pt * t_pt * spp_eq) / (e_nrc * t_nrc)
    st = mlp.state()
    # MLP inference throughput on the frame's 2.07M cache queries
    n = W_PX * H_PX
    out = torch.zeros(n * 3, dtype=torch.float32, device=dev)
    for _ in range(3):
        mlp.inference(r.infer, out, n)
    torch.cuda.synchronize()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record()
    for _ in range(10):
        mlp.inference(r.infer, out, n)
    q1.record()
    q1.synchronize()
    t_inf = q0.elapsed_time(q1) / 10
    flops = 2.0 * (96 * 64 + 4 * 64 * 64 + 64 * 16) * n

    # Inference-precision sweep on the trained cache: the same frame (same
    # paths, no further training) answered in FP16, BF16 and FP8 (E4M3 with
    # per-layer scales calibrated on the last frame's queries).
    from tfg_b200.nrc import BF16, FP8, FP16
    r.cfg.train_steps = 0
    mlp.calibrate(r.infer, n, stream=r.stream)
    sweep = {}
    for name, prec in (("fp16", FP16), ("bf16", BF16), ("fp8", FP8)):
        mlp.set_precision(prec)
        r.frame(40_000, accumulate=False)
        r.stream.synchronize()
        img_p = r.image().cpu().numpy().astype(np.float64)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(r.stream)
        for k in range(10):
            r.frame(40_000, accumulate=False)
        f1.record(r.stream)
        f1.synchronize()
        with torch.cuda.stream(r.stream):
            for _ in range(3):
                mlp.inference(r.infer, out, n, stream=r.stream)
            g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            g0.record(r.stream)
            for _ in range(10):
                mlp.inference(r.infer, out, n, stream=r.stream)
            g1.record(r.stream)
        g1.synchronize()
        ti = g0.elapsed_time(g1) / 10
        sweep[name] = {"relmse": round(rel(img_p), 5), "ms_per_frame_no_training": round(f0.elapsed_time(f1) / 10, 3),
                       "inference_ms": round(ti, 4), "inference_tflops_fp16_equiv": round(flops / (ti * 1e-3) / 1e12, 1)}
    mlp.set_precision(FP16)
    mlp.close()

    # Depth and encoding sweeps: the same protocol (warm-up, orbit, final
    # pose) with 3 and 7 hidden layers of 64 (5 is the run above), and with
    # the reference's own input encoding (hash grid + one-blob + identity).
    def variant(fp8: bool = False, **kw) -> dict:
        m2 = ColorMLP(batch=16384, seed=2024, **kw)
        m2.set_bounds(*scene.bounds)
        r2 = NrcRenderer(ds, m2, params, train_steps=4, use_graph=True)
        for f in range(48):
            with torch.cuda.stream(r2.stream):
                set_pose(0)
            r2.frame(f, warmup=True, accumulate=False)
        for k in range(frames):
            with torch.cuda.stream(r2.stream):
                set_pose(k)
            r2.frame(48 + k, accumulate=False)
        d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        d0.record(r2.stream)
        for k in range(10):
            r2.frame(10_000 + k, accumulate=False)
        d1.record(r2.stream)
        d1.synchronize()
        img2 = r2.image().cpu().numpy().astype(np.float64)
        with torch.cuda.stream(r2.stream):
            for _ in range(3):
                m2.inference(r2.infer, out, n, stream=r2.stream)
            h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            h0.record(r2.stream)
            for _ in range(10):
                m2.inference(r2.infer, out, n, stream=r2.stream)
            h1.record(r2.stream)
        h1.synchronize()
        if fp8:
            # the trained cache answered in FP8 (scales calibrated on the last frame's queries)
            m2.calibrate(r2.infer, n, stream=r2.stream)
            m2.set_precision(FP8)
            r2.cfg.train_steps = 0
            r2.frame(40_000, accumulate=False)
            r2.stream.synchronize()
            img8 = r2.image().cpu().numpy().astype(np.float64)
            with torch.cuda.stream(r2.stream):
                for _ in range(3):
                    m2.inference(r2.infer, out, n, stream=r2.stream)
                k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                k0.record(r2.stream)
                for _ in range(10):
                    m2.inference(r2.infer, out, n, stream=r2.stream)
                k1.record(r2.stream)
            k1.synchronize()
            fp8_res = {"relmse": round(rel(img8), 5), "inference_ms": round(k0.elapsed_time(k1) / 10, 4)}
            m2.set_precision(FP16)
        res = {"relmse": round(rel(img2), 5), "ms_per_frame": round(d0.elapsed_time(d1) / 10, 3),
               "inference_ms": round(h0.elapsed_time(h1) / 10, 4), "adam_steps": int(m2.state()["adam_t"]),
               "loss_ema": round(m2.state()["loss_ema"], 5)}
        if fp8:
            res["fp8"] = fp8_res
        m2.close()
        return res

    # Cache-policy sweep: the reference's termination policy (footprint 0.01
    # of render.h:102, 5 % training paths of render.h:443, the first diffuse
    # vertex past the footprint) against variants, each from a fresh model
    # through the same protocol, scored at equal GPU time against the same
    # 4096-spp reference.
    plain_rel = {spp_eq: e_pt}

    def plain_at(spp: int) -> float:
        if spp not in plain_rel:
            img_p = pt.accumulate_spp(ds, params, spp, 30_000).cpu().numpy().astype(np.float64)
            plain_rel[spp] = rel(img_p)
        return plain_rel[spp]

    def policy(footprint=0.01, train_fraction=0.05, train_steps=4, hidden_layers=5, gate=0.0) -> dict:
        m3 = ColorMLP(batch=16384, seed=2024, hidden_layers=hidden_layers)
        m3.set_bounds(*scene.bounds)
        r3 = NrcRenderer(ds, m3, params, train_steps=train_steps, use_graph=True, footprint=footprint,
                         train_fraction=train_fraction, gate_threshold=gate)
        for f in range(48):
            with torch.cuda.stream(r3.stream):
                set_pose(0)
            r3.frame(f, warmup=True, accumulate=False)
        for k in range(frames):
            with torch.cuda.stream(r3.stream):
                set_pose(k)
            r3.frame(48 + k, accumulate=False)
        d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        d0.record(r3.stream)
        for k in range(10):
            r3.frame(10_000 + k, accumulate=False)
        d1.record(r3.stream)
        d1.synchronize()
        t3 = d0.elapsed_time(d1) / 10
        e3 = rel(r3.image().cpu().numpy().astype(np.float64))
        answered = float((r3.thr.view(-1, 3) != 0).any(dim=1).float().mean())
        sp = max(1, int(round(t3 / t_pt)))
        ep = plain_at(sp)
        out3 = {"footprint": footprint, "train_fraction": round(train_fraction, 5), "train_steps": train_steps,
                "hidden_layers": hidden_layers, "gate_threshold": gate, "relmse": round(e3, 5),
                "ms_per_frame": round(t3, 3), "plain_spp_at_equal_time": sp, "relmse_plain": round(ep, 5),
                "relmse_ratio_plain_over_nrc": round(ep / e3, 3),
                "relmse_x_time_ratio": round((ep * t_pt * sp) / (e3 * t3), 3),
                "pixels_answered_by_cache": round(answered, 4)}
        if gate > 0:
            out3["open_gate_cells"] = int(m3.state()["gate"])
        m3.close()
        return out3

    one_per_record = 65536 / n   # about as many training paths as records a frame uses
    sweep_defs = {
        "reference": {},
        "footprint_0.001": {"footprint": 0.001},
        "footprint_0.1": {"footprint": 0.1},
        "primary_vertex": {"footprint": 0.0},
        "train_fraction_3.2pct": {"train_fraction": one_per_record},
        "train_steps_1": {"train_steps": 1},
        "train_steps_2": {"train_steps": 2},
        "3x64": {"hidden_layers": 3},
        "primary_vertex_train_3.2pct": {"footprint": 0.0, "train_fraction": one_per_record},
        "primary_vertex_train_3.2pct_steps_2": {"footprint": 0.0, "train_fraction": one_per_record, "train_steps": 2},
        "gated_0.5": {"gate": 0.5},
        "primary_vertex_gated_0.5": {"footprint": 0.0, "train_fraction": one_per_record, "gate": 0.5},
    }
    policy_sweep = {name: policy(**kw) for name, kw in sweep_defs.items()}
    best = max(policy_sweep, key=lambda k: policy_sweep[k]["relmse_x_time_ratio"])

    depth = {5: {"relmse": round(e_nrc, 5), "ms_per_frame": round(t_nrc, 3), "inference_ms": round(t_inf, 4),
                 "adam_steps": int(st["adam_t"])}}
    for hidden in (3, 7):
        depth[hidden] = variant(hidden_layers=hidden)
    from tfg_b200.nrc import HASHGRID, hashgrid_reference
    encoding = {"frequency_12_bands": depth[5],
                "hashgrid_reference": {**variant(encoding=HASHGRID), "config": hashgrid_reference(),
                                       "one_blob_bins": 4}}
    width = {"5x64": depth[5], "5x128": variant(fp8=True, width=128), "3x128": variant(hidden_layers=3, width=128),
             "7x128": variant(hidden_layers=7, width=128)}
    return {
        "frames": 48 + frames, "warmup_frames": 48, "camera": "orbit 1 deg/frame", "train_samples_per_frame": 4 * 16384,
        "ms_per_frame_nrc": round(t_nrc, 3), "ms_per_pass_plain_1spp": round(t_pt, 3),
        "plain_spp_at_equal_time": spp_eq, "relmse_nrc": round(e_nrc, 5), "relmse_plain": round(e_pt, 5),
        "tuning": tuning_1spp.__dict__,
        "relmse_ratio_plain_over_nrc": round(e_pt / e_nrc, 3), "relmse_x_time_ratio": round(ratio_time, 3),
        "reference_spp": ref_spp, "adam_steps": int(st["adam_t"]), "loss_ema": round(st["loss_ema"], 5),
        "mlp_inference": {"queries": n, "ms": round(t_inf, 4), "tflops": round(flops / (t_inf * 1e-3) / 1e12, 2),
                          "flops_per_query": int(flops / n)},
        "policy_sweep": policy_sweep,
        "best_policy": {"name": best, **policy_sweep[best]},
        # the target: at least 2x lower relMSE than plain path tracing given the same GPU time
        "target_2x_lower_relmse_at_equal_time": {
            "met": policy_sweep[best]["relmse_ratio_plain_over_nrc"] >= 2.0, "policy": best,
            "relmse_ratio_plain_over_nrc": policy_sweep[best]["relmse_ratio_plain_over_nrc"],
            "relmse_x_time_ratio": policy_sweep[best]["relmse_x_time_ratio"]},
        "precision_sweep": sweep,
        "depth_sweep": {f"{k}x64": v for k, v in sorted(depth.items())},
        "encoding_sweep": encoding,
        "width_sweep": width,
    }


def c1_eval(dev, nthreads: int) -> dict:
    """The reference's CPU-runnable case (config 1): displaced icosphere
    (subdiv 6, 81,920 tris) in a 12-triangle box, one light, 512x512, 16 spp,
    depth 5, roulette from depth 3, frames 1..16.  GPU time with resident
    inputs, the CPU oracle on all host cores for the same 16 samples, and the
    relMSE between the two images (same RNG streams)."""
    import ctypes

    import numpy as np
    import torch

    from oracle import oracle as orc
    from tfg_b200 import bvh as hbvh
    from tfg_b200 import pathtracer as pt
    from tfg_b200 import scenes
    s = scenes.box_icosphere(512, 512, subdiv=6, seed=1)
    ds = pt.DeviceScene(s, dev)
    W, H, spp = s.width, s.height, 16
    p = pt.RenderParams(max_depth=5, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT, spp=spp,
                        accumulate=1)
    acc = torch.zeros(W * H * 3, device=dev)
    tuning, _ = pt.autotune(ds, p, repeats=3)
    for _ in range(3):
        acc.zero_()
        pt.render_pass(ds, p, 1, None, acc)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 10
    e0.record()
    for _ in range(reps):
        acc.zero_()
        pt.render_pass(ds, p, 1, None, acc)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    gpu_img = (acc / spp).view(H, W, 3).cpu().numpy().astype(np.float64)
    ds.close()
    hb = hbvh.build_host(hbvh.triangle_vertices(s.mesh))
    prm = pt.RenderParams(max_depth=5, rr_min_depth=3, shadow_mesh=1).c()
    cpu = np.zeros((H, W, 3), np.float64)
    img = np.zeros((H, W, 3), np.float32)
    t0 = time.perf_counter()
    for f in range(1, spp + 1):
        orc.cpu.orc_render(orc.p(s.prims), len(s.prims), orc.p(s.lights), len(s.lights), orc.p(hb.nodes),
                           orc.p(hb.tris_ref), orc.p(s.mesh), len(s.mesh), orc.p(s.camera), W, H, f,
                           ctypes.addressof(prm), 0, H, orc.p(img), None, None, None, None, 0, 0, nthreads)
        cpu += img
    t_cpu = time.perf_counter() - t0
    cpu /= spp
    relmse = float(np.mean((gpu_img - cpu) ** 2 / (cpu ** 2 + 1e-2)))
    return {"workload": "512x512, 16 spp, depth 5, RR from 3, displaced icosphere (81,920 tris) in a 12-tri box, "
                        "1 light, frames 1..16",
            "gpu_ms_per_frame": round(ms, 3), "gpu_mpaths_per_s": round(W * H * spp / (ms * 1e-3) / 1e6, 1),
            "tuning": tuning.__dict__,
            "cpu_s_per_frame": round(t_cpu, 2), "cpu_mpaths_per_s": round(W * H * spp / t_cpu / 1e6, 3),
            "cpu_cores": nthreads, "cpu_kind": "port",
            "relmse_gpu_vs_cpu_oracle": relmse, "note": "the CPU oracle uses the reference's transform triangle "
            "test, the GPU the watertight one"}


def batched_eval(dev, frames: int = 20) -> dict:
    """Twelve independent scenes (10k to 2M triangles, 1-4 lights, 640x360 to
    1920x1080), one cache model each, 1 spp + cache per frame, advanced by
    one tfgNrcFrameBatch call per frame and replayed as one CUDA graph.  Also
    times the same batch without the graph and the twelve scenes as
    single-scene tfgNrcFrame calls one after another."""
    import torch

    from tfg_b200 import pathtracer as pt
    from tfg_b200 import scenes as sc
    from tfg_b200.nrc import ColorMLP, NrcBatch, NrcRenderer

    params = pt.RenderParams(max_depth=DEPTH, rr_min_depth=RR, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)
    t0 = time.perf_counter()
    scs = [sc.batch_scene(i) for i in range(12)]
    dss = [pt.DeviceScene(s, dev) for s in scs]
    t_setup = time.perf_counter() - t0
    rs = []
    for k, (s, ds) in enumerate(zip(scs, dss)):
        m = ColorMLP(batch=16384, seed=500 + k)
        m.set_bounds(*s.bounds)
        rs.append(NrcRenderer(ds, m, params, train_steps=4, use_graph=True))
    batch = NrcBatch(rs, use_graph=True)
    st = batch.stream
    for f in range(48):
        batch.frame(f, warmup=True)
    for f in range(8):
        batch.frame(48 + f)
    st.synchronize()
    # Autotuned queue and MLP tile sizes: the launch settings on the largest
    # scene (plain 1-spp passes), the model's tiling on that scene's cache
    # queries; every model shares the architecture and takes the same tiling.
    big = max(range(len(scs)), key=lambda k: scs[k].width * scs[k].height)
    render_tuning, _ = pt.autotune(dss[big], params, repeats=3, stream=st)
    n_big = scs[big].width * scs[big].height
    scratch = torch.zeros(n_big * 3, dtype=torch.float32, device=dev)
    mlp_tuning = rs[big].mlp.autotune(rs[big].infer, scratch, n_big, repeats=5, stream=st)
    for r in rs:
        r.mlp.set_tuning(mlp_tuning["wgrad_tiles_per_cta"], mlp_tuning["infer_ctas"])
    batch.frame(56)   # captures the graph again under the new settings
    st.synchronize()

    def timed(fn, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for k in range(n):
            fn(k)
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / n

    ms_graph = timed(lambda k: batch.frame(1000 + k), frames)
    eager = NrcBatch(rs, use_graph=False, stream=st)
    ms_eager = timed(lambda k: eager.frame(2000 + k), frames)

    # tfgNrcFrame keeps one captured graph per device, so twelve alternating
    # scenes run as eager single-scene calls
    for r in rs:
        r.stream = st
        r.cfg.use_graph = 0

    def one_by_one(k):
        for r in rs:
            r.frame(3000 + k, accumulate=False)

    one_by_one(0)
    ms_single = timed(one_by_one, frames)
    px = sum(s.width * s.height for s in scs)
    adam = [int(r.mlp.state()["adam_t"]) for r in rs]
    for r in rs:
        r.mlp.close()
    for ds in dss:
        ds.close()
    return {
        "scenes": len(scs), "triangles": [int(len(s.mesh)) for s in scs],
        "resolutions": [f"{s.width}x{s.height}" for s in scs], "lights": [int(len(s.lights)) for s in scs],
        "paths_per_frame": px, "frames_timed": frames,
        "ms_per_batch_frame_graph": round(ms_graph, 3), "ms_per_batch_frame_eager": round(ms_eager, 3),
        "ms_per_frame_12_single_scene_calls": round(ms_single, 3),
        "mpaths_per_s_graph": round(px / (ms_graph * 1e-3) / 1e6, 1),
        "adam_steps_min": min(adam), "setup_s": round(t_setup, 1),
        "render_tuning": render_tuning.__dict__, "mlp_tuning": mlp_tuning,
        "frame": "render 1 spp with cache queries + training records, inference + composite, targets, 4 Adam steps",
    }


def compare_bvh_builders():
    """Host binned-SAH builder (tfgTinyBVHConstruir) against the device
    Morton-order builder (tfgTinyBVHConstruirGPU) on the benchmark scene:
    build time (including the primitive upload; the second of two builds, so
    that module loading and first allocations stay out), primary-ray
    throughput and 8-spp path throughput with each tree."""
    import torch

    from tfg_b200 import pathtracer as pt
    from tfg_b200 import scenes
    s = scenes.spheres_terrain(W_PX, H_PX)
    n = W_PX * H_PX
    out = {}
    for name, gpu in (("host_sah", False), ("device_morton", True)):
        pt.DeviceScene(s, "cuda", gpu_build=gpu).close()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ds = pt.DeviceScene(s, "cuda", gpu_build=gpu)
        torch.cuda.synchronize()
        tb = time.perf_counter() - t0
        rays = torch.empty(n * 8, device="cuda")
        hits = torch.empty(n * 4, device="cuda")
        pt.camera_rays(ds, 0, rays)
        for _ in range(3):
            pt.trace_rays(ds, rays, hits, pt.TRIS_WATERTIGHT)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            pt.trace_rays(ds, rays, hits, pt.TRIS_WATERTIGHT)
        e1.record()
        torch.cuda.synchronize()
        grays = n * 10 / (e0.elapsed_time(e1) * 1e-3) / 1e9
        p = pt.RenderParams(max_depth=DEPTH, rr_min_depth=RR, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT, spp=8,
                            accumulate=1)
        acc = torch.zeros(n * 3, device="cuda")
        pt.render_pass(ds, p, 0, None, acc)
        torch.cuda.synchronize()
        e0.record()
        pt.render_pass(ds, p, 100, None, acc)
        e1.record()
        torch.cuda.synchronize()
        out[name] = {"build_s_incl_upload": round(tb, 3), "nodes": int(ds.bvh.ref.num_nodos),
                     "depth": int(ds.bvh.max_depth), "primary_grays_per_s": round(grays, 3),
                     "mpaths_per_s_8spp": round(n * 8 / (e0.elapsed_time(e1) * 1e-3) / 1e6, 1)}
        ds.close()
    print(json.dumps(out))


def measure_peaks():
    """Peaks this pod's MEASURED_PEAKS.json does not hold, measured the same
    way (best of 10, CUDA events): an L2-resident copy (2 x 24 MB buffers,
    read + write bytes), and dense FP16 and FP8 (e4m3, per-tensor scales)
    GEMMs of 8192^3 through torch (cuBLAS / cuBLASLt)."""
    import torch
    dev = torch.device("cuda", 0)

    def best_ms(fn, reps=10):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    out = {}
    n = 24 << 20
    a = torch.empty(n, dtype=torch.uint8, device=dev).fill_(1)
    b = torch.empty(n, dtype=torch.uint8, device=dev)
    inner = 50
    ms = best_ms(lambda: [b.copy_(a) for _ in range(inner)])
    out["l2_copy_gbs"] = round(2 * n * inner / (ms * 1e-3) / 1e9, 1)
    big = 1 << 30
    a2 = torch.empty(big, dtype=torch.uint8, device=dev).fill_(1)
    b2 = torch.empty(big, dtype=torch.uint8, device=dev)
    ms = best_ms(lambda: b2.copy_(a2))
    out["hbm_copy_gbs"] = round(2 * big / (ms * 1e-3) / 1e9, 1)
    del a2, b2
    N = 8192
    x = torch.randn(N, N, device=dev, dtype=torch.float16)
    y = torch.randn(N, N, device=dev, dtype=torch.float16)
    ms = best_ms(lambda: torch.matmul(x, y))
    out["fp16_tflops"] = round(2 * N ** 3 / (ms * 1e-3) / 1e12, 1)
    xb, yb = x.bfloat16(), y.bfloat16()
    ms = best_ms(lambda: torch.matmul(xb, yb))
    out["bf16_tflops"] = round(2 * N ** 3 / (ms * 1e-3) / 1e12, 1)
    try:
        x8 = x.to(torch.float8_e4m3fn)
        y8 = y.t().contiguous().t().to(torch.float8_e4m3fn)
        one = torch.ones((), device=dev)
        ms = best_ms(lambda: torch._scaled_mm(x8, y8, scale_a=one, scale_b=one, out_dtype=torch.bfloat16))
        out["fp8_e4m3_tflops"] = round(2 * N ** 3 / (ms * 1e-3) / 1e12, 1)
    except Exception as e:   # older torch without the scaled GEMM
        out["fp8_e4m3_tflops"] = None
        out["fp8_error"] = str(e).splitlines()[0][:200]
    out["how"] = ("best of 10 CUDA-event timings after 3 warm-ups; L2: 50 back-to-back copies of a 24 MB buffer; "
                  "HBM: one 1 GiB copy; GEMMs: torch.matmul / torch._scaled_mm, 8192^3, 2*N^3 FLOP")
    print(json.dumps(out))


def profile_mlp(width: int = 64, precision: str = "fp16"):
    """Cache inference over 2,073,600 queries (232 MB of DatosMLP, more than
    L2) and one 16384-sample train step of a network of 5 hidden layers of
    `width` units, untimed; used for ncu captures.  With precision "fp8" the
    FP16 inference is preceded by a calibration pass and two FP8 inferences."""
    import numpy as np
    import torch

    from tfg_b200.nrc import FP8, FP16, ColorMLP
    from tfg_b200.structs import DATOS_MLP
    n = W_PX * H_PX
    rng = np.random.default_rng(0)
    d = np.zeros(n, DATOS_MLP)
    for k in "xyz":
        d["posicion"][k] = rng.uniform(-5, 5, n)
        d["direccion"][k] = rng.uniform(0, 1, n)
        d["normal"][k] = rng.uniform(0, 1, n)
    for k in "rgb":
        d["difuso"][k] = rng.uniform(0, 1, n)
        d["color"][k] = rng.uniform(0, 2, n)
    dd = torch.from_numpy(d.view(np.uint8).copy()).cuda()
    m = ColorMLP(batch=16384, seed=1, width=width)
    m.set_bounds((-6, -6, -6), (6, 6, 6))
    out = torch.zeros(n * 3, device="cuda")
    if precision == "fp8":
        m.set_precision(FP8)
        m.calibrate(dd, n)
        for _ in range(2):
            m.inference(dd, out, n)
        m.set_precision(FP16)
    m.inference(dd, out, n)
    m.train_step(dd, n, read_loss=False)
    torch.cuda.synchronize()
    m.close()
    print("profile mlp done")


def profile_train(width: int = 64, steps: int = 30):
    """`steps` eager training steps of 16,384 samples (5 hidden layers of
    `width` units, frequency encoding) drawn from 65,536 seeded records, then
    exit; the case for a warm launch list of the step's kernels (k_train,
    k_wgrad, k_adam): skip the first steps' launches in ncu."""
    import numpy as np
    import torch

    from tfg_b200.nrc import ColorMLP
    from tfg_b200.structs import DATOS_MLP
    n = 65536
    rng = np.random.default_rng(0)
    d = np.zeros(n, DATOS_MLP)
    for k in "xyz":
        d["posicion"][k] = rng.uniform(-5, 5, n)
        d["direccion"][k] = rng.uniform(0, 1, n)
        d["normal"][k] = rng.uniform(0, 1, n)
    for k in "rgb":
        d["difuso"][k] = rng.uniform(0, 1, n)
        d["color"][k] = rng.uniform(0, 2, n)
    dd = torch.from_numpy(d.view(np.uint8).copy()).cuda()
    m = ColorMLP(batch=16384, seed=1, width=width)
    m.set_bounds((-6, -6, -6), (6, 6, 6))
    for _ in range(steps):
        m.train_step(dd, n, read_loss=False)
    torch.cuda.synchronize()
    m.close()
    print("profile train done")


def profile_frame(encoding: str = "frequency", width: int = 64, frames: int = 6, footprint: float = 0.01):
    """`frames` cache frames of the 1920x1080 benchmark scene (the first
    four as warm-up frames, 4 x 16384 training samples each, launched
    eagerly) and then one more inference over the last frame's 2,073,600
    queries, untimed; used for ncu launch lists and captures.  Every frame
    launches `k_infer` twice (the frame's queries and the tail queries), so
    the last inference is launch 2 * frames of that kernel."""
    import torch

    from tfg_b200 import pathtracer as pt
    from tfg_b200 import scenes
    from tfg_b200.nrc import HASHGRID, ColorMLP, NrcRenderer
    scene = scenes.spheres_terrain(W_PX, H_PX)
    ds = pt.DeviceScene(scene, "cuda")
    params = pt.RenderParams(max_depth=DEPTH, rr_min_depth=RR, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT)
    kw = {"encoding": HASHGRID} if encoding == "hashgrid" else {}
    m = ColorMLP(batch=16384, seed=2024, width=width, **kw)
    m.set_bounds(*scene.bounds)
    r = NrcRenderer(ds, m, params, train_steps=4, use_graph=False, footprint=footprint)
    for f in range(frames):
        r.frame(f, warmup=f < 4, accumulate=False)
    n = W_PX * H_PX
    out = torch.zeros(n * 3, dtype=torch.float32, device="cuda")
    with torch.cuda.stream(r.stream):
        m.inference(r.infer, out, n, stream=r.stream)
    r.stream.synchronize()
    m.close()
    ds.close()
    print("profile frame done")


def profile_pass(samples: int = 1, tuning: str | None = None):
    """One pass of `samples` spp (8 bounces) of the benchmark frame in one
    wavefront of samples x W x H paths: ~0.3 GB of scene data (more than L2)
    and ~0.5 GB of queues per sample; used for ncu captures.  `tuning`: JSON
    object of further TfgRenderTuning fields (e.g. the autotuner's pick)."""
    import torch

    from tfg_b200 import pathtracer as pt
    from tfg_b200 import scenes
    scene = scenes.spheres_terrain(W_PX, H_PX)
    ds = pt.DeviceScene(scene, "cuda")
    fields = {"wavefront_paths": 0 if samples == 1 else samples * W_PX * H_PX, **json.loads(tuning or "{}")}
    pt.set_tuning(pt.RenderTuning(**fields))
    p = pt.RenderParams(max_depth=DEPTH, rr_min_depth=RR, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT,
                        spp=samples, accumulate=1)
    accum = torch.zeros(W_PX * H_PX * 3, dtype=torch.float32, device="cuda")
    pt.render_pass(ds, p, 1, None, accum)
    torch.cuda.synchronize()
    ds.close()
    print("profile pass done")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-nrc", action="store_true", help="skip the radiance-cache evaluation")
    ap.add_argument("--no-batched", action="store_true", help="skip the 12-scene batched cache frame")
    ap.add_argument("--profile-pass", action="store_true",
                    help="run one untimed pass of the workload and exit (small case for ncu)")
    ap.add_argument("--wavefront-samples", type=int, default=1,
                    help="with --profile-pass: samples per pass, all in one wavefront")
    ap.add_argument("--tuning", default=None,
                    help='with --profile-pass: JSON of launch tuning fields, e.g. \'{"shadow_one_lane": 1}\'')
    ap.add_argument("--compare-bvh-builders", action="store_true",
                    help="host SAH vs device Morton-order CWBVH: build time and traversal speed, then exit")
    ap.add_argument("--measure-peaks", action="store_true",
                    help="measure L2 copy bandwidth and FP16 / BF16 / FP8 GEMM peaks, print them and exit")
    ap.add_argument("--profile-mlp", action="store_true",
                    help="run cache inference on 1920x1080 queries and one train step, then exit (case for ncu)")
    ap.add_argument("--mlp-width", type=int, default=64,
                    help="with --profile-mlp / --profile-frame: 64 or 128 units per hidden layer")
    ap.add_argument("--mlp-precision", default="fp16", choices=["fp16", "fp8"],
                    help="with --profile-mlp: fp8 adds a calibration pass and two FP8 inferences")
    ap.add_argument("--profile-train", action="store_true",
                    help="run 30 eager 16,384-sample training steps of the cache model, then exit (case for ncu)")
    ap.add_argument("--profile-frame", action="store_true",
                    help="run six eager cache frames of the workload and one more inference, then exit (case for ncu)")
    ap.add_argument("--mlp-encoding", default="frequency", choices=["frequency", "hashgrid"],
                    help="with --profile-frame: the cache's input encoding")
    ap.add_argument("--nrc-footprint", type=float, default=0.01,
                    help="with --profile-frame: the cache policy's footprint threshold (0: query at the primary hit)")
    ap.add_argument("--nrc-only", action="store_true",
                    help="run only the radiance-cache evaluation (config 3 and its sweeps), print it and exit")
    args = ap.parse_args()
    if args.nrc_only:
        import torch

        from tfg_b200 import pathtracer as pt
        from tfg_b200 import scenes
        scene = scenes.spheres_terrain(W_PX, H_PX)
        ds = pt.DeviceScene(scene, "cuda")
        print(json.dumps(nrc_eval(scene, ds, torch.device("cuda", 0))))
        ds.close()
        return
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.profile_pass:
        profile_pass(args.wavefront_samples, args.tuning)
        return
    if args.profile_frame:
        profile_frame(args.mlp_encoding, args.mlp_width, footprint=args.nrc_footprint)
        return
    if args.profile_mlp:
        profile_mlp(args.mlp_width, args.mlp_precision)
        return
    if args.profile_train:
        profile_train(args.mlp_width)
        return
    if args.measure_peaks:
        measure_peaks()
        return
    if args.compare_bvh_builders:
        compare_bvh_builders()
        return

    import torch

    from tfg_b200 import pathtracer as pt
    from tfg_b200 import scenes

    rank, world, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scene = scenes.spheres_terrain(W_PX, H_PX)
    ds = pt.DeviceScene(scene, dev)
    n_px = W_PX * H_PX
    base = pt.RenderParams(max_depth=DEPTH, rr_min_depth=RR, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT,
                           spp=SPP, accumulate=1)
    accum = torch.zeros(n_px * 3, dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2
    stream = torch.cuda.current_stream()

    # Traversal work per ray (outside the timed region): one 1-spp pass with counters.
    pt.profile_reset()
    cnt_params = pt.RenderParams(**{**base.__dict__, "spp": 1, "profile": pt.PROFILE_COUNTS})
    pt.render_pass(ds, cnt_params, 999, None, accum)
    work = pt.profile_get()
    rays_per_spp = work["rays"]
    nodes_per_ray = work["nodes"] / max(1, work["rays"])
    tris_per_ray = work["tri_tests"] / max(1, work["rays"])
    # Algorithmic bytes of one closest-hit ray (watertight layout): 80 B per node
    # decoded, 48 B per triangle tested, 32 B ray read, 16 B hit written.
    bytes_per_ray = 80.0 * nodes_per_ray + 48.0 * tris_per_ray + 32.0 + 16.0
    # The same for a shadow ray (any hit): nodes and triangles, its share of the
    # 64 B shading-point item and of the 16 B radiance update.
    shadow_per_spp = work["shadow_rays"]
    shadow_nodes = work["shadow_nodes"] / max(1, work["shadow_rays"])
    shadow_tris = work["shadow_tri_tests"] / max(1, work["shadow_rays"])
    shadow_bytes = 80.0 * shadow_nodes + 48.0 * shadow_tris + 64.0 + 16.0

    # The autotuner picks the wavefront size and launch shapes on this frame
    # (untimed, like the warm-up); the timed frames and the e2e calls use it.
    t_tune = time.perf_counter()
    tuning, tune_table = pt.autotune(ds, base, repeats=3)
    tune_s = time.perf_counter() - t_tune
    tuned_ms = min(ms for t, ms in tune_table if t == tuning)

    for s in range(args.warmup):
        accum.zero_()
        pt.render_pass(ds, base, 1000 * (s + 1), None, accum)
    torch.cuda.synchronize()

    timed = pt.RenderParams(**{**base.__dict__, "profile": pt.PROFILE_TIMES})
    pt.profile_reset()
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record(stream)
        for s in range(args.steps):
            flush.fill_(s & 0xFF)
            accum.zero_()
            pt.render_pass(ds, timed, replica_frame(rank, s, args.steps), None, accum)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    prof = pt.profile_get()
    ms_max = max_over_ranks(ms, world)
    paths = n_px * SPP * args.steps
    value = replicas_value(paths, ms_max, world)

    # End to end through the C ABI with host buffers: per frame, camera + lights
    # from pinned host memory, 64-spp render, accumulated image back to pinned host.
    cam_h = torch.from_numpy(scene.camera.view("u1").copy()).pin_memory()
    lig_h = torch.from_numpy(scene.lights.view("u1").copy()).pin_memory()
    img_h = torch.empty(n_px * 3, dtype=torch.float32).pin_memory()
    e2e_steps = max(1, min(args.steps, 3))
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s in range(e2e_steps):
        ds.camera.copy_(cam_h, non_blocking=True)
        ds.lights.copy_(lig_h, non_blocking=True)
        accum.zero_()
        pt.render_pass(ds, base, 7 + SPP * s, None, accum)
        img_h.copy_(accum, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
    wall_ms = (time.perf_counter() - t0) * 1e3
    e2e_value = world * n_px * SPP * e2e_steps / (e2e_ms * 1e-3) / 1e6

    # Primary-ray traversal throughput (rays resident in HBM) through the
    # traversal-only entry: the primary rays of as many samples per call as
    # the tuned wavefront holds, in the path tracer's 8 x 4 tile order, and
    # one sample per call (scanline and tile order) for comparison.
    def primary(samples: int, order: int, reps: int = 10) -> float:
        rays = torch.empty(samples * n_px * 8, dtype=torch.float32, device=dev)
        hits = torch.empty(samples * n_px * 4, dtype=torch.float32, device=dev)
        pt.camera_rays_ex(ds, 0, samples, order, rays)
        for _ in range(3):
            pt.trace_rays(ds, rays, hits, pt.TRIS_WATERTIGHT)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(reps):
            pt.trace_rays(ds, rays, hits, pt.TRIS_WATERTIGHT)
        p1.record(stream)
        torch.cuda.synchronize()
        del rays, hits
        return samples * n_px * reps / (p0.elapsed_time(p1) * 1e-3) / 1e9

    primary_samples = max(1, min(16, tuning.wavefront_paths // n_px)) if tuning.wavefront_paths else 1
    primary_grays = primary(primary_samples, pt.RAYS_TILES)
    primary_one = {"scanline": round(primary(1, pt.RAYS_SCANLINE), 3), "tiles": round(primary(1, pt.RAYS_TILES), 3)}

    if rank != 0:
        ds.close()
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    nrc = None
    if not args.no_nrc and world == 1:
        nrc = nrc_eval(scene, ds, dev)
        bf16 = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()).get("bf16_tflops") if (ROOT / "MEASURED_PEAKS.json").exists() else 1590.0
        nrc["mlp_inference"]["frac_of_dense_f16_peak"] = round(nrc["mlp_inference"]["tflops"] / bf16, 4)
        nrc["mlp_inference"]["peak_tflops"] = bf16

    batched = None
    if not args.no_batched and world == 1:
        batched = batched_eval(dev)
    c1 = None
    if not args.no_cpu_baseline and world == 1:
        c1 = c1_eval(dev, os.cpu_count() or 1)

    pk = peaks()
    trace_ms = prof["ms"]["trace"]
    trace_launches = prof["launches"]["trace"]
    rays_timed = rays_per_spp * SPP * args.steps
    achieved = rays_timed * bytes_per_ray / (trace_ms * 1e-3) / 1e9 if trace_ms > 0 else None
    l2_achieved = (rays_timed * TRACE_L2_BYTES_PER_RAY / (trace_ms * 1e-3) / 1e9
                   if trace_ms > 0 and TRACE_L2_BYTES_PER_RAY else None)
    l2_peak = l2_gather_peak(dev)
    shadow_ms = prof["ms"]["shadow"]
    shadow_timed = shadow_per_spp * SPP * args.steps
    shadow_achieved = shadow_timed * shadow_bytes / (shadow_ms * 1e-3) / 1e9 if shadow_ms > 0 else None
    launches = sum(prof["launches"].values())
    clocks = clk.summary()

    cpu = None
    if not args.no_cpu_baseline:
        from tfg_b200 import bvh as hbvh
        hb = hbvh.build_host(hbvh.triangle_vertices(scene.mesh))
        nthreads = os.cpu_count() or 1
        # full frames at 1 spp until at least 12 s of CPU work (at most 64)
        frames, dt, n = 0, 0.0, 0
        while dt < 12.0 and frames < 64:
            d, k = cpu_oracle_sample(scene, hb, H_PX, nthreads, frame=1 + frames)
            dt += d
            n += k
            frames += 1
        cpu = {"value": round(n / dt / 1e6, 4), "unit": "Mpaths/s", "cores": nthreads, "kind": "port",
               "sample": f"{frames} full 1920x1080 frames at 1 spp ({frames} of the 64 samples of the timed frame; "
                         f"depth {DEPTH}, RR from {RR}), {dt:.1f} s"}

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
        "config": {"workload": WORKLOAD, "width": W_PX, "height": H_PX, "spp_per_frame": SPP,
                   "max_depth": DEPTH, "rr_min_depth": RR, "triangles": int(ds.n_mesh),
                   "tri_test": "watertight", "parallelism": f"replicas x{world}",
                   "l2": "flushed between steps (256 MB write); scene inputs (200 MB primitives + 64 MB CWBVH) exceed L2"},
        "ms_per_frame_1spp": round(ms_max / args.steps / SPP, 3),
        "e2e": {"value": round(e2e_value, 3), "unit": "Mpaths/s", "h2d_bytes_per_step": 112 + 80,
                "d2h_bytes_per_step": n_px * 12, "ms_per_step": round(e2e_ms / e2e_steps, 3),
                "wall_ms_per_step": round(wall_ms / e2e_steps, 3), "call": "tfgRenderPass"},
        "roofline": {
            "kernel": "k_trace (CWBVH closest hit)", "bound": "hbm",
            # What limits k_trace: its scene is L2-resident and it is issue-bound with half of each
            # warp's lanes active (divergent node counts per ray); the HBM fraction above is the
            # contract's figure, the L2 and issue fractions below say how far the kernel is from a roof.
            "limiter": "instruction issue with divergent lanes (L2-resident scene)",
            "l2_gbs": round(l2_achieved, 1) if l2_achieved else None,
            "l2_peak_gbs": l2_peak["gbs"], "l2_peak_how": l2_peak["how"],
            "l2_frac": round(l2_achieved / l2_peak["gbs"], 4) if l2_achieved else None,
            "l2_bytes_per_ray": TRACE_L2_BYTES_PER_RAY,
            "issue_frac": TRACE_ISSUE_FRAC, "simt_efficiency": TRACE_SIMT_EFFICIENCY,
            "achieved": round(achieved, 1) if achieved else None,
            "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": round(achieved / pk["hbm_gbs"], 4) if achieved else None,
            "peak_source": pk["source"],
            # ncu dram__bytes_read.sum + dram__bytes_write.sum per closest-hit ray (eight launches of
            # one pass, 1- and 16-sample wavefronts) times this run's rays per launch: the 64 MB CWBVH +
            # triangles stay L2-resident, so DRAM sees ~6-8 % of the algorithmic bytes.
            "traffic": trace_traffic(tuning.wavefront_paths, n_px, rays_timed / max(1, trace_launches)),
            "traffic_unit": "bytes per launch",
            "algorithmic_bytes_per_ray": round(bytes_per_ray, 1),
            "nodes_per_ray": round(nodes_per_ray, 3), "tri_tests_per_ray": round(tris_per_ray, 3),
            "rays_per_launch_avg": round(rays_timed / max(1, trace_launches), 1),
            "ms_per_launch_avg": round(trace_ms / max(1, trace_launches), 4),
            "stage_ms": {k: round(v, 2) for k, v in prof["ms"].items()},
        },
        # The shadow stage takes as much device time as the closest-hit one (launch list in
        # profiles/launches_bench_1080p_64spp.md); its figures on the same terms.  Its CUDA-event
        # time runs on the side stream beside the next bounce's trace, so `achieved` is low by
        # the share of the GPU that trace holds meanwhile.
        "roofline_shadow": {
            "kernel": "k_shadow (CWBVH any hit, one lane per shading point)", "bound": "hbm",
            "limiter": "instruction issue with divergent lanes (L2-resident scene)",
            "simt_efficiency": SHADOW_SIMT_EFFICIENCY,
            "achieved": round(shadow_achieved, 1) if shadow_achieved else None,
            "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": round(shadow_achieved / pk["hbm_gbs"], 4) if shadow_achieved else None,
            "algorithmic_bytes_per_ray": round(shadow_bytes, 1),
            "nodes_per_ray": round(shadow_nodes, 3), "tri_tests_per_ray": round(shadow_tris, 3),
            "rays_timed": shadow_timed, "ms": round(shadow_ms, 2),
        },
        "primary_rays": {"grays_per_s": round(primary_grays, 3), "rays_per_call": primary_samples * n_px,
                         "samples_per_call": primary_samples, "order": "8x4 tiles", "tri_test": "watertight",
                         "grays_per_s_one_sample_per_call": primary_one,
                         "hit_ids_vs_reference": "checked bit for bit against the reference traverse_cwbvh on these "
                                                 "1080p camera rays (4 frames, reference triangle layout) by "
                                                 "tests/test_gpu_fullsize.py::"
                                                 "test_primary_ids_bit_exact_vs_reference_traversal_1080p; the "
                                                 "timed region runs only the drop-in",
                         "note": "a call of one sample (2,073,600 rays) waits on its few longest grazing rays; "
                                 "more samples per call amortise that tail"},
        "autotune": {
            "tuning": tuning.__dict__, "seconds": round(tune_s, 2), "spp_per_pass": min(SPP, 16),
            "pass_ms_start": round(tune_table[0][1], 3), "pass_ms_tuned": round(tuned_ms, 3),
            "candidates": [[t.wavefront_paths, t.trace_threads, t.trace_warps_per_sm, t.refill_min,
                            t.shadow_one_lane, t.refill_min_primary, t.overlap_shadow, round(ms, 3)]
                           for t, ms in tune_table],
            "candidate_fields": ["wavefront_paths", "trace_threads", "trace_warps_per_sm", "refill_min",
                                 "shadow_one_lane", "refill_min_primary", "overlap_shadow", "ms_per_pass"],
        },
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "nrc": nrc,
        "batched": batched,
        "c1_cpu_runnable_case": c1,
    }
    print(json.dumps(out))
    ds.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
