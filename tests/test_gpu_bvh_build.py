"""The device CWBVH builder (tfgTinyBVHConstruirGPU) against the host builder
and brute force: same primitive hand-off (TRIANGULO entries in input order),
every triangle in exactly one leaf, closest hits equal to brute force and to
the host-built tree (up to equal-distance ties), and the same images."""
import time

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from tests.helpers import rel_mse
from tfg_b200 import bvh as hbvh
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes
from tfg_b200.devmem import view_device
from tfg_b200.structs import PRIMITIVA, TRIANGULO

pytestmark = pytest.mark.gpu
MISS = 0xFFFFFFFF


def _random_rays(rng, n, lo, hi):
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 3] = 1e9
    return r


def _trace(ds, rays, fmt):
    dr = torch.from_numpy(rays.reshape(-1).copy()).cuda()
    hits = torch.zeros(len(rays) * 4, dtype=torch.float32, device="cuda")
    pt.trace_rays(ds, dr, hits, fmt)
    torch.cuda.synchronize()
    return hits.view(-1, 4).cpu().numpy()


def _check_structure(ds, scene):
    b = ds.bvh
    tri_mask = scene.mesh["tipo"] == TRIANGULO
    nt = int(tri_mask.sum())
    assert b.num_primitivas == nt and b.ref.num_tris == nt
    prims = view_device(b.d_primitivas, nt * PRIMITIVA.itemsize, np.uint8).cpu().numpy()
    np.testing.assert_array_equal(prims, np.ascontiguousarray(scene.mesh[tri_mask]).view(np.uint8))
    wt = view_device(b.d_tris_wt, nt * 12).cpu().numpy().reshape(nt, 12)
    ids = wt[:, 3].view(np.uint32)
    assert sorted(ids.tolist()) == list(range(nt))           # each triangle in exactly one leaf
    ref = view_device(b.ref.d_tris, nt * 16).cpu().numpy().reshape(nt, 16)
    np.testing.assert_array_equal(ref[:, 15].view(np.uint32), ids)
    assert 1 <= b.max_depth <= 64


def _mesh_of(tris):
    m = np.zeros(len(tris), PRIMITIVA)
    m["tipo"] = TRIANGULO
    m["u"][:, :9] = np.asarray(tris, np.float64).reshape(len(tris), 9)
    return m


@pytest.mark.parametrize("case", ["one", "two", "duplicates", "mixed"])
def test_small_and_degenerate_inputs(built, case):
    rng = np.random.default_rng(5)
    base = scenes.tiny_box(32, 32, subdiv=1)
    if case == "one":
        mesh = _mesh_of([[-1, -1, 2, 1, -1, 2, 0, 1, 2]])
    elif case == "two":
        mesh = _mesh_of([[-1, -1, 2, 1, -1, 2, 0, 1, 2], [-1, -1, 3, 1, -1, 3, 0, 1, 3]])
    elif case == "duplicates":   # many triangles on one centroid: equal Morton codes
        t = rng.normal(size=(1, 9)) * 0.3
        mesh = _mesh_of(np.repeat(t, 50, axis=0) + rng.normal(size=(50, 9)) * 1e-7)
    else:                        # analytic spheres interleaved with the triangles: ids follow the compaction
        tri = base.mesh[base.mesh["tipo"] == TRIANGULO]
        sph = scenes.sphere_prim((0.0, 0.0, 3.0), 0.5)
        mesh = np.concatenate([sph, tri[:7], sph, tri[7:], sph])
    s = scenes.Scene(base.prims, mesh, base.lights, base.camera, base.width, base.height, bounds=base.bounds,
                     name=case)
    ds = pt.DeviceScene(s, "cuda", gpu_build=True)
    _check_structure(ds, s)
    hb = hbvh.build_host(hbvh.triangle_vertices(mesh))
    rays = _random_rays(rng, 4000, [-2, -2, -1], [2, 2, 5])
    got = _trace(ds, rays, pt.TRIS_REF)
    want = orc.brute_batch(hb.tris_ref, rays)
    a, b = got[:, 3].view(np.uint32), want[:, 3].view(np.uint32)
    hit = b != MISS
    np.testing.assert_array_equal(a != MISS, hit)
    if case != "duplicates":     # coincident triangles tie at equal t
        np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(got[hit, 0], want[hit, 0], rtol=1e-5)
    ds.close()


@pytest.fixture(scope="module")
def pair(built):
    s = scenes.spheres_terrain(160, 96, subdiv=3, terrain_n=120)
    host = pt.DeviceScene(s, "cuda")
    gpu = pt.DeviceScene(s, "cuda", gpu_build=True)
    yield s, host, gpu
    host.close()
    gpu.close()


def test_structure_and_hits_match_host_build(pair):
    s, host, gpu = pair
    _check_structure(gpu, s)
    rng = np.random.default_rng(7)
    rays = _random_rays(rng, 30000, [-10, -1.5, -18], [10, 3, 2])
    cam = torch.zeros(s.width * s.height * 8, device="cuda")
    pt.camera_rays(host, 1, cam)
    rays = np.concatenate([rays, cam.view(-1, 8).cpu().numpy()]).astype(np.float32)
    for fmt in (pt.TRIS_REF, pt.TRIS_WATERTIGHT):
        a = _trace(gpu, rays, fmt)
        b = _trace(host, rays, fmt)
        ia, ib = a[:, 3].view(np.uint32), b[:, 3].view(np.uint32)
        assert (ia != ib).mean() < 1e-3, (fmt, (ia != ib).mean())   # equal-t ties may resolve differently
        both = (ia == ib) & (ia != MISS)
        np.testing.assert_array_equal(a[both, 0], b[both, 0])


def test_images_match_host_build(pair):
    s, host, gpu = pair
    p = pt.RenderParams(max_depth=6, rr_min_depth=3, shadow_mesh=1, tri_format=pt.TRIS_WATERTIGHT, spp=4,
                        accumulate=1)
    imgs = []
    for ds in (host, gpu):
        acc = torch.zeros(s.width * s.height * 3, device="cuda")
        pt.render_pass(ds, p, 11, None, acc)
        torch.cuda.synchronize()
        imgs.append(acc.cpu().numpy() / 4)
    assert rel_mse(imgs[1], imgs[0]) <= 1e-4


def test_million_triangle_build_time(built):
    s = scenes.spheres_terrain(64, 64)             # 1,000,480 triangles
    t0 = time.perf_counter()
    ds = pt.DeviceScene(s, "cuda", gpu_build=True)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    _check_structure(ds, s)
    print(f"device build of {ds.n_mesh} triangles (with upload): {dt * 1e3:.1f} ms, "
          f"{ds.bvh.ref.num_nodos} nodes, depth {ds.bvh.max_depth}")
    ds.close()
