"""The composite encoding of the oracle (hash grid + one-blob + identity):
properties that pin it without a GPU -- index ranges, dense levels as a
bijection, one-blob bins, and the table gradient against finite differences
of the encoding (which is linear in the table values)."""
import numpy as np

from oracle import mlp_oracle as mo

CFG = {"n_levels": 6, "log2_hashmap_size": 12, "base_resolution": 4.0, "per_level_scale": 2.0}


def test_reference_levels():
    levels, T = mo.hashgrid_levels({"n_levels": 16, "log2_hashmap_size": 19, "base_resolution": 16.0,
                                    "per_level_scale": 1.5})
    assert T == 2 ** 19
    assert [N for N, _ in levels][:6] == [16, 24, 36, 54, 81, 121]
    assert [d for _, d in levels] == [True] * 4 + [False] * 12


def test_indices_in_range_and_dense_levels_bijective():
    levels, T = mo.hashgrid_levels(CFG)
    for N, dense in levels:
        g = np.arange(N + 1, dtype=np.uint64)
        x, y, z = np.meshgrid(g, g, g, indexing="ij")
        q = mo.hash_index(x.ravel(), y.ravel(), z.ravel(), N, dense, T)
        assert q.max() < T
        if dense:
            assert len(np.unique(q)) == (N + 1) ** 3


def test_one_blob_bins():
    rng = np.random.default_rng(0)
    r15 = rng.uniform(0, 1, (400, 15)).astype(np.float32)
    r15[0, 3:9] = 0.0
    r15[1, 3:9] = 1.0
    levels, T = mo.hashgrid_levels(CFG)
    x, _ = mo.composite_encode(r15, np.zeros(len(levels) * T * 2), CFG)
    blob = x[:, 32:56].reshape(-1, 6, 4)
    assert (blob >= 0).all() and (blob.sum(-1) <= 1 + 1e-12).all()
    # mirror symmetry: the bins of s are the bins of 1 - s reversed
    r2 = r15.copy()
    r2[:, 3:9] = 1.0 - r15[:, 3:9]
    x2, _ = mo.composite_encode(r2, np.zeros(len(levels) * T * 2), CFG)
    np.testing.assert_allclose(x2[:, 32:56].reshape(-1, 6, 4)[..., ::-1], blob, atol=1e-6)
    assert (x[:, 62] == 1.0).all() and (x[:, 63:] == 0).all()
    np.testing.assert_array_equal(x[:, 56:62], r15[:, 9:15])


def test_table_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    levels, T = mo.hashgrid_levels(CFG)
    size = len(levels) * T * 2
    tab = rng.uniform(-1, 1, size)
    r15 = rng.uniform(0, 1, (64, 15)).astype(np.float32)
    L2 = 2 * len(levels)
    c = rng.normal(size=(64, L2))                 # objective: sum(c * features)
    x, corners = mo.composite_encode(r15, tab, CFG)
    g = mo.table_grad(c, corners, size)
    # the features are linear in the table: grad . delta == change of the objective
    for _ in range(5):
        delta = rng.normal(size=size) * 1e-3
        x2, _ = mo.composite_encode(r15, tab + delta, CFG)
        np.testing.assert_allclose(np.sum(c * (x2[:, :L2] - x[:, :L2])), g @ delta, rtol=1e-9, atol=1e-12)


def test_corner_weights_sum_to_one():
    rng = np.random.default_rng(2)
    r15 = rng.uniform(0, 1, (100, 15)).astype(np.float32)
    r15[:3, :3] = [[0, 0, 0], [1, 1, 1], [0.5, 1, 0]]
    _, corners = mo.composite_encode(r15, np.zeros(6 * 4096 * 2), CFG)
    for lst in corners:
        np.testing.assert_allclose(sum(w for _, w in lst), 1.0, atol=1e-6)
