"""Primary-ray traversal parity on the GPU.

The product traversal (tfgTraceRays) runs on the same CWBVH as the
reference's own traverse_cwbvh (compiled from the reference sources into
oracle/_ref) and as the CPU restatement.  With the reference triangle layout
the closest-hit ids must agree bit for bit; with the watertight test they
must agree except on genuine edge hits, with t within 1e-5 relative."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from tfg_b200 import bvh as hbvh
from tfg_b200 import pathtracer as pt
from tfg_b200 import scenes

pytestmark = pytest.mark.gpu

MISS = 0xFFFFFFFF


@pytest.fixture(scope="module")
def setup(built):
    scene = scenes.box_icosphere(256, 192, subdiv=5)
    ds = pt.DeviceScene(scene, "cuda")
    W, H = scene.width, scene.height
    rays = torch.zeros(W * H * 8, dtype=torch.float32, device="cuda")
    pt.camera_rays(ds, 3, rays)
    # plus incoherent rays from inside the box
    rng = np.random.default_rng(0)
    n = 60000
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = rng.uniform([-2.5, -1.9, -3.9], [2.5, 2.3, 5.4], (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 3] = 1e9
    rays_all = torch.cat([rays, torch.from_numpy(r.reshape(-1)).cuda()])
    yield scene, ds, rays, rays_all
    ds.close()


def _trace(ds, rays, fmt):
    hits = torch.zeros(rays.numel() // 2, dtype=torch.float32, device="cuda")
    pt.trace_rays(ds, rays, hits, fmt)
    torch.cuda.synchronize()
    return hits.view(-1, 4).cpu().numpy()


def _ref_trace(ds, rays):
    ref = orc.ref()
    if ref is None:
        pytest.skip("reference kernels (oracle/_ref) not built")
    n = rays.numel() // 8
    hits = torch.zeros(n * 4, dtype=torch.float32, device="cuda")
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert ref.ref_trace(ds.bvh.ref.d_nodos, ds.bvh.ref.d_tris, rays.data_ptr(), n, hits.data_ptr(),
                         steps.data_ptr()) == 0
    torch.cuda.synchronize()
    return hits.view(-1, 4).cpu().numpy(), steps.cpu().numpy()


def test_camera_rays_match_cpu_restatement(setup):
    scene, ds, rays, _ = setup
    got = rays.view(-1, 8).cpu().numpy()
    want = orc.camera_rays(scene.camera, scene.width, scene.height, 3)
    np.testing.assert_allclose(got[:, :7], want[:, :7], rtol=0, atol=2e-7)
    assert (got[:, :7] == want[:, :7]).mean() > 0.999


def test_ref_layout_ids_bit_exact_vs_reference_traversal(setup):
    _, ds, _, rays = setup
    mine = _trace(ds, rays, pt.TRIS_REF)
    ref, _ = _ref_trace(ds, rays)
    a, b = mine[:, 3].view(np.uint32), ref[:, 3].view(np.uint32)
    assert (a != MISS).mean() > 0.05
    assert np.array_equal(a, b), f"{(a != b).sum()} id mismatches"
    hit = a != MISS
    np.testing.assert_allclose(mine[hit, 0], ref[hit, 0], rtol=1e-6)
    np.testing.assert_allclose(mine[hit, 1:3], ref[hit, 1:3], rtol=1e-5, atol=1e-6)


def test_axis_plane_rays_keep_the_reference_hits(setup):
    # Directions with exactly zero components (either sign of zero) take a
    # finite reciprocal of that zero's sign in the slab tests (the reference's
    # 1/0 = infinity gives 0 * infinity = NaN, which switches that axis' box
    # culling off and made one bench camera ray decode 382 nodes instead of
    # 7).  A ray with a signed-zero component is thereby treated as moving
    # infinitesimally to that side.  The ids must equal the reference's except
    # for rays lying exactly in a plane through mesh edges (here: origin x = 0,
    # the icosphere's symmetry plane), and there only on the reference's edge
    # hits, where the side the reference found depended on its disabled culling.
    scene, ds, _, _ = setup
    rng = np.random.default_rng(3)
    n = 40000
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = rng.uniform([-2.5, -1.9, -3.9], [2.5, 2.3, 5.4], (n, 3))
    d = rng.normal(size=(n, 3))
    k = rng.integers(0, 3, n)
    d[np.arange(n), k] = 0.0
    d[rng.random(n) < 0.25] *= np.array([0.0, 1.0, 0.0])[None, :]   # some rays along y only
    d[(d == 0).all(1)] = [0.0, -1.0, 0.0]
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    d[rng.random((n, 3)) < 0.5] *= -1.0                                # -0.0 as well as +0.0
    r[:, 4:7] = d
    r[:, 3] = 1e9
    r[: n // 4, 0] = 0.0                                                # in the symmetry plane x = 0
    assert ((r[:, 4:7] == 0) & np.signbit(r[:, 4:7])).any() and ((r[:, 4:7] == 0) & ~np.signbit(r[:, 4:7])).any()
    rays = torch.from_numpy(r.reshape(-1)).cuda()
    mine = _trace(ds, rays, pt.TRIS_REF)
    ref, _ = _ref_trace(ds, rays)
    a, b = mine[:, 3].view(np.uint32), ref[:, 3].view(np.uint32)
    assert (a != MISS).sum() > 1000          # the icosphere mesh (the box walls are analytic)
    bad = a != b
    in_plane = (r[:, 0] == 0.0) & (r[:, 4] == 0.0)
    assert not (bad & ~in_plane).any(), f"{(bad & ~in_plane).sum()} mismatches off the symmetry plane"
    u, v = ref[:, 1], ref[:, 2]
    ref_on_edge = (b != MISS) & (np.minimum(np.minimum(u, v), 1.0 - u - v) < 1e-6)
    assert (ref_on_edge | ~bad).all()
    assert bad.mean() < 1e-3
    same = ~bad & (a != MISS)
    np.testing.assert_allclose(mine[same, 0], ref[same, 0], rtol=1e-6)


def test_watertight_ids_vs_reference_traversal(setup):
    scene, ds, _, rays = setup
    mine = _trace(ds, rays, pt.TRIS_WATERTIGHT)
    ref, _ = _ref_trace(ds, rays)
    a, b = mine[:, 3].view(np.uint32), ref[:, 3].view(np.uint32)
    same = a == b
    # mismatches must be edge / vertex hits: a barycentric within 1e-4 of an edge in
    # either result, or both hits at the same distance (adjacent triangles)
    def near_edge(h):
        u, v = h[:, 1], h[:, 2]
        return np.minimum(np.minimum(u, v), 1.0 - u - v) < 1e-4
    tie = np.isclose(mine[:, 0], ref[:, 0], rtol=1e-5) & (a != MISS) & (b != MISS)
    explained = near_edge(mine) | near_edge(ref) | tie
    bad = ~same & ~explained
    assert bad.sum() == 0, f"{bad.sum()} unexplained id mismatches of {len(a)}"
    assert (~same).mean() < 1e-3
    both = same & (a != MISS)
    rel = np.abs(mine[both, 0] - ref[both, 0]) / ref[both, 0]
    assert np.quantile(rel, 0.99) <= 1e-5, f"t rel error p99 {np.quantile(rel, 0.99):.2e}"
    assert rel.max() <= 1e-3, f"t rel error {rel.max():.2e}"
    # Where the two disagree by more than 1e-5, the exact (FP64) distance to the
    # same triangle decides: the watertight t must be the accurate one.  The
    # reference's plane-row test t = -(T2.O + w) / (T2.D) loses precision at
    # grazing incidence (T2.D -> 0).
    hb = hbvh.build_host(hbvh.triangle_vertices(scene.mesh))
    r = rays.view(-1, 8).cpu().numpy().astype(np.float64)
    tri_of = np.empty(hb.num_tris, np.int64)
    tri_of[hb.tris_wt[:, 3].view(np.uint32)] = np.arange(hb.num_tris)
    k = np.nonzero(both)[0]
    v = hb.tris_wt[tri_of[a[k]]].astype(np.float64)
    v0, v1, v2 = v[:, 0:3], v[:, 4:7], v[:, 8:11]
    n = np.cross(v1 - v0, v2 - v0)
    t_exact = np.einsum("ij,ij->i", v0 - r[k, 0:3], n) / np.einsum("ij,ij->i", r[k, 4:7], n)
    err_wt = np.abs(mine[k, 0] - t_exact) / t_exact
    err_ref = np.abs(ref[k, 0] - t_exact) / t_exact
    assert np.quantile(err_wt, 0.9999) <= 1e-5, f"watertight t vs exact: {np.quantile(err_wt, 0.9999):.2e}"
    off = rel > 1e-5
    assert (err_wt[off] <= err_ref[off]).all()


def test_traversal_vs_cpu_oracle(setup):
    scene, ds, _, rays = setup
    hb = hbvh.build_host(hbvh.triangle_vertices(scene.mesh))
    mine = _trace(ds, rays, pt.TRIS_REF)
    cpu, _ = orc.trace_batch(hb.nodes, hb.tris_ref, rays.view(-1, 8).cpu().numpy())
    a, b = mine[:, 3].view(np.uint32), cpu[:, 3].view(np.uint32)
    assert (a != b).mean() < 1e-4
    both = (a == b) & (a != MISS)
    rel = np.abs(mine[both, 0] - cpu[both, 0]) / cpu[both, 0]
    # The oracle rounds every operation (no FMA contraction); the device
    # contracts multiply-adds.  They differ only through the grazing-angle
    # sensitivity of the reference plane test.
    assert np.quantile(rel, 0.999) <= 1e-5 and rel.max() <= 1e-3


def test_device_bvh_equals_host_build(setup):
    """tfgTinyBVHConstruir uploads exactly what tfgCWBVHBuild returns."""
    scene, ds, _, _ = setup
    hb = hbvh.build_host(hbvh.triangle_vertices(scene.mesh))
    assert ds.bvh.ref.num_nodos == hb.num_nodes and ds.bvh.ref.num_tris == hb.num_tris
    from tfg_b200.devmem import view_device
    nodes = view_device(ds.bvh.ref.d_nodos, hb.nodes.size).cpu().numpy()
    tris = view_device(ds.bvh.ref.d_tris, hb.tris_ref.size).cpu().numpy()
    wt = view_device(ds.bvh.d_tris_wt, hb.tris_wt.size).cpu().numpy()
    assert np.array_equal(tris.view(np.uint32), hb.tris_ref.reshape(-1).view(np.uint32))
    assert np.array_equal(wt.view(np.uint32), hb.tris_wt.reshape(-1).view(np.uint32))
    assert np.array_equal(nodes.view(np.uint32), hb.nodes.reshape(-1).view(np.uint32))


def test_empty_batch_and_all_miss(setup):
    _, ds, _, _ = setup
    r = torch.zeros(8 * 64, dtype=torch.float32, device="cuda").view(64, 8)
    r[:, 0:3] = 100.0        # far outside, pointing away
    r[:, 4] = 1.0
    r[:, 3] = 1e9
    h = _trace(ds, r.reshape(-1), pt.TRIS_WATERTIGHT)
    assert (h[:, 3].view(np.uint32) == MISS).all() and (h[:, 0] == 1e9).all()
    pt.trace_rays(ds, torch.zeros(0, device="cuda"), torch.zeros(0, device="cuda"))


def test_camera_rays_in_samples_and_tile_order(setup):
    scene, ds, _, _ = setup
    W, H = scene.width, scene.height
    n = W * H
    single = []
    for f in range(5, 8):
        r = torch.zeros(n * 8, device="cuda")
        pt.camera_rays(ds, f, r)
        single.append(r.view(-1, 8))
    lin = torch.zeros(3 * n * 8, device="cuda")
    pt.camera_rays_ex(ds, 5, 3, pt.RAYS_SCANLINE, lin)
    til = torch.zeros(3 * n * 8, device="cuda")
    pt.camera_rays_ex(ds, 5, 3, pt.RAYS_TILES, til)
    torch.cuda.synchronize()
    perm = torch.from_numpy(pt.tiled_pixels(W, H)).cuda()
    for s in range(3):
        assert torch.equal(lin.view(-1, 8)[s * n:(s + 1) * n], single[s])
        assert torch.equal(til.view(-1, 8)[s * n:(s + 1) * n], single[s][perm])
    # tile order hits the same primitives as scanline order, ray for ray
    hl, ht = _trace(ds, lin, pt.TRIS_WATERTIGHT), _trace(ds, til, pt.TRIS_WATERTIGHT)
    p3 = np.concatenate([perm.cpu().numpy() + s * n for s in range(3)])
    assert np.array_equal(ht[:, 3].view(np.uint32), hl[p3, 3].view(np.uint32))
