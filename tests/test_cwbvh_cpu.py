"""CWBVH builder checks on the CPU: the node encoding decodes to a valid tree
and the reference traversal (CPU restatement of traverse_cwbvh.cuh) finds the
same closest hit as a brute-force loop over every triangle."""
import numpy as np
import pytest

from tfg_b200 import bvh as hbvh
from tfg_b200 import scenes


def _random_rays(rng, n, lo=-2.0, hi=2.0):
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = o
    r[:, 3] = 1e9
    r[:, 4:7] = d
    return r


def _decode(hb):
    """Walk the tree from the node words; return (#nodes reached, triangle refs)."""
    nodes = hb.nodes.view(np.uint32)
    seen, tri_refs = set(), []
    stack = [0]
    while stack:
        i = stack.pop()
        assert i not in seen
        seen.add(i)
        w = nodes[i]
        imask = int(w[3] >> 24)
        child_base, tri_base = int(w[4]), int(w[5])
        meta = w[6:8].view(np.uint8)
        rel = 0
        for s in range(8):
            m = int(meta[s])
            if imask & (1 << s):
                assert (m & 0x1F) == 24 + s and (m >> 5) == 1
                stack.append(child_base + rel)
                rel += 1
            elif m:
                cnt = {1: 1, 3: 2, 7: 3}[m >> 5]
                off = m & 0x1F
                assert off + cnt <= 24
                tri_refs.extend(tri_base // 4 + off + k for k in range(cnt))
    return len(seen), tri_refs


@pytest.mark.parametrize("subdiv", [0, 1, 3])
def test_tree_covers_every_triangle_once(subdiv):
    s = scenes.box_icosphere(16, 16, subdiv=subdiv)
    hb = hbvh.build_host(hbvh.triangle_vertices(s.mesh))
    n_nodes, refs = _decode(hb)
    assert n_nodes == hb.num_nodes
    assert sorted(refs) == list(range(hb.num_tris))
    ids = np.sort(hb.tris_ref[:, 15].view(np.uint32))
    assert (ids == np.arange(len(s.mesh))).all()
    # both triangle layouts are in the same order
    assert (hb.tris_ref[:, 15].view(np.uint32) == hb.tris_wt[:, 3].view(np.uint32)).all()


@pytest.mark.parametrize("n", [2, 3, 4, 5, 7, 9, 10, 24, 25, 64])
def test_small_and_coincident_triangle_sets(n):
    # the 8-wide collapse on tiny trees (leaves of up to 3 triangles, nodes of
    # 2..8 slots) and on triangles that all share one centroid (split by index)
    from oracle import oracle as orc
    rng = np.random.default_rng(n)
    c = rng.uniform(-1.0, 1.0, (n, 1, 3))
    v = (c + rng.uniform(-0.3, 0.3, (n, 3, 3))).astype(np.float32)
    same = np.repeat(rng.uniform(-0.3, 0.3, (1, 3, 3)), n, axis=0)
    same[:, 0] += np.linspace(-1e-3, 1e-3, n)[:, None]
    same[:, 1] -= np.linspace(-1e-3, 1e-3, n)[:, None]           # the centroids stay equal
    for verts in (v, same.astype(np.float32)):
        hb = hbvh.build_host(verts.reshape(-1, 9))
        n_nodes, refs = _decode(hb)
        assert n_nodes == hb.num_nodes and sorted(refs) == list(range(n))
        rays = _random_rays(rng, 3000, -1.5, 1.5)
        got, _ = orc.trace_batch(hb.nodes, hb.tris_ref, rays)
        want = orc.brute_batch(hb.tris_ref, rays)
        a, b = got[:, 3].view(np.uint32), want[:, 3].view(np.uint32)
        assert (a == b).all()


@pytest.mark.parametrize("subdiv,n_rays", [(2, 4000), (4, 6000)])
def test_traversal_matches_brute_force(subdiv, n_rays):
    from oracle import oracle as orc
    rng = np.random.default_rng(subdiv)
    s = scenes.box_icosphere(16, 16, subdiv=subdiv)
    hb = hbvh.build_host(hbvh.triangle_vertices(s.mesh))
    rays = _random_rays(rng, n_rays)
    hits, counts = orc.trace_batch(hb.nodes, hb.tris_ref, rays)
    brute = orc.brute_batch(hb.tris_ref, rays)
    ids, bids = hits[:, 3].view(np.uint32), brute[:, 3].view(np.uint32)
    assert (ids != 0xFFFFFFFF).mean() > 0.05
    assert (ids == bids).all()
    assert np.array_equal(hits[:, 0], brute[:, 0])
    assert counts[:, 0].min() >= 1


def test_camera_rays_hit_like_brute_force():
    from oracle import oracle as orc
    s = scenes.box_icosphere(48, 32, subdiv=3)
    hb = hbvh.build_host(hbvh.triangle_vertices(s.mesh))
    rays = orc.camera_rays(s.camera, 48, 32, frame=5)
    hits, _ = orc.trace_batch(hb.nodes, hb.tris_ref, rays)
    brute = orc.brute_batch(hb.tris_ref, rays)
    assert (hits[:, 3].view(np.uint32) == brute[:, 3].view(np.uint32)).all()


def test_degenerate_and_duplicate_triangles():
    from oracle import oracle as orc
    rng = np.random.default_rng(11)
    tri = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32)
    verts = np.concatenate([
        np.repeat(tri, 40, axis=0),                                   # 40 identical triangles (all centroids equal)
        np.array([[0, 0, 0, 1, 1, 1, 2, 2, 2]], np.float32),           # zero-area (collinear)
        np.array([[5, 5, 5, 5, 5, 5, 5, 5, 5]], np.float32),           # a point
        rng.uniform(-1, 1, (200, 9)).astype(np.float32),
    ])
    hb = hbvh.build_host(verts)
    n_nodes, refs = _decode(hb)
    assert sorted(refs) == list(range(len(verts)))
    rays = _random_rays(rng, 3000, -1.5, 1.5)
    hits, _ = orc.trace_batch(hb.nodes, hb.tris_ref, rays)
    brute = orc.brute_batch(hb.tris_ref, rays)
    a, b = hits[:, 3].view(np.uint32), brute[:, 3].view(np.uint32)
    assert np.array_equal(hits[:, 0], brute[:, 0])
    # identical duplicates tie exactly; which of them wins depends on visit order
    tie = (a < 40) & (b < 40)
    assert (a[~tie] == b[~tie]).all()
    # the degenerate triangles are never reported
    deg = {40, 41}
    assert not deg & set(hits[:, 3].view(np.uint32).tolist())


def test_single_triangle_known_answer():
    from oracle import oracle as orc
    verts = np.array([[0, 0, -2, 1, 0, -2, 0, 1, -2]], np.float32)
    hb = hbvh.build_host(verts)
    r = np.zeros((3, 8), np.float32)
    r[:, 3] = 1e9
    r[:, 6] = -1.0
    r[0, :3] = (0.25, 0.25, 0.0)     # hits at t=2, u=0.25, v=0.25
    r[1, :3] = (0.8, 0.8, 0.0)       # outside (u+v > 1)
    r[2, :3] = (0.25, 0.25, -3.0)    # triangle behind the origin
    hits, _ = orc.trace_batch(hb.nodes, hb.tris_ref, r, nthreads=1)
    assert hits[0, 3].view(np.uint32) == 0
    np.testing.assert_allclose(hits[0, :3], [2.0, 0.25, 0.25], rtol=1e-6)
    assert hits[1, 3].view(np.uint32) == 0xFFFFFFFF and hits[2, 3].view(np.uint32) == 0xFFFFFFFF


def test_large_coordinates_and_flat_scene():
    """Quantisation exponents for a far-away, perfectly flat mesh."""
    from oracle import oracle as orc
    rng = np.random.default_rng(2)
    # 16 x 16 grid of quads (512 non-overlapping triangles) on the plane z = 500
    g = np.linspace(1000.0, 1010.0, 17)
    tris = []
    for i in range(16):
        for j in range(16):
            a, b = (g[i], g[j]), (g[i + 1], g[j])
            c, d = (g[i], g[j + 1]), (g[i + 1], g[j + 1])
            tris.append([*a, 500, *b, 500, *c, 500])
            tris.append([*b, 500, *d, 500, *c, 500])
    verts = np.array(tris, np.float32)
    hb = hbvh.build_host(verts)
    r = np.zeros((2000, 8), np.float32)
    r[:, 0:2] = rng.uniform(1000.0, 1010.0, (2000, 2))
    r[:, 2] = 0.0
    r[:, 3] = 1e9
    r[:, 6] = 1.0
    hits, _ = orc.trace_batch(hb.nodes, hb.tris_ref, r)
    brute = orc.brute_batch(hb.tris_ref, r)
    assert (hits[:, 3].view(np.uint32) == brute[:, 3].view(np.uint32)).all()
    assert (hits[:, 3].view(np.uint32) != 0xFFFFFFFF).mean() > 0.5
