"""The CPU oracle against golden outputs of the reference's own GPU kernels
(tests/golden/*.npz, written by tests/golden/make_golden.py from
RenderKernel.cu / NrcKernel.cu compiled unmodified).  This pins the oracle
without a GPU: traversal hits (traverse_cwbvh.cuh:51-257), path-traced
images (kernelRender_tiny, RenderKernel.cu:19-47), the element-wise NRC
kernels (RenderKernel.cu:49-166, NrcKernel.cu:5-126) and the default camera.
Tolerances are those of the GPU parity tests: the reference kernels contract
multiply-adds on the device, the oracle rounds every operation."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as orc
from tests.helpers import oracle_image, rel_mse
from tfg_b200 import bvh as hbvh
from tfg_b200 import scenes
from tfg_b200.structs import BOUNDS, CAMARA, COLOR, DATOS_MLP, REGISTRO

GOLD = Path(__file__).resolve().parent / "golden"
MISS = 0xFFFFFFFF


def _load(name):
    p = GOLD / name
    if not p.exists():
        pytest.fail(f"missing golden fixture {p} (python tests/golden/make_golden.py on a GPU machine)")
    return np.load(p)


def _host_bvh(scene, g):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", GOLD / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    hb = hbvh.build_host(hbvh.triangle_vertices(scene.mesh))
    assert mg.bvh_hash(hb) == str(g["bvh_sha256"]), "the BVH builder changed: regenerate the golden fixtures"
    return hb, mg


@pytest.mark.parametrize("name", ["reference_room", "tiny_box"])
def test_oracle_images_match_reference_kernel(name):
    g = _load(f"render_{name}.npz")
    scene = {"reference_room": lambda: scenes.reference_room(32, 32, subdiv=2),
             "tiny_box": lambda: scenes.tiny_box(32, 32, subdiv=2)}[name]()
    hb, _ = _host_bvh(scene, g)
    for f, ref_img in zip(g["frames"], g["images"]):
        img = oracle_image(orc, scene, hb, int(f))
        assert np.isfinite(img).all()
        assert rel_mse(img, ref_img) <= 1e-4, (name, int(f), rel_mse(img, ref_img))


def test_oracle_traversal_matches_reference_kernel():
    g = _load("trace_box_icosphere.npz")
    scene = scenes.box_icosphere(64, 48, subdiv=3)
    hb, mg = _host_bvh(scene, g)
    rays = g["rays"]
    np.testing.assert_array_equal(rays, mg.trace_rays_input(scene))     # same seeded inputs
    cpu, _ = orc.trace_batch(hb.nodes, hb.tris_ref, rays)
    ref = g["hits"]
    a, b = cpu[:, 3].view(np.uint32), ref[:, 3].view(np.uint32)
    assert (a != b).sum() <= 2, int((a != b).sum())
    assert (b != MISS).mean() > 0.05
    both = (a == b) & (a != MISS)
    rel = np.abs(cpu[both, 0] - ref[both, 0]) / ref[both, 0]
    assert np.quantile(rel, 0.999) <= 1e-5 and rel.max() <= 1e-3


def test_oracle_nrc_kernels_match_reference_kernels():
    # Every array handed to the oracle is bound to a name first: NpzFile
    # materialises a new array per access, and a temporary's buffer would be
    # freed before the C call runs.
    g = dict(_load("nrc_kernels.npz"))
    img = g["comp_img"].copy()
    orc.cpu.orc_composite(orc.p(img), orc.p(g["comp_pred"]), orc.p(g["comp_thr"]), len(img))
    np.testing.assert_allclose(img, g["comp_out"], rtol=1e-6, atol=1e-6)

    regs = g["regs"].view(REGISTRO)
    n = len(regs)
    tgt = np.zeros(n, DATOS_MLP)
    orc.cpu.orc_targets(orc.p(regs), orc.p(g["tail"]), orc.p(tgt), n)
    want = g["targets"].view(DATOS_MLP)
    for f in ("posicion", "direccion", "normal"):
        for k in "xyz":
            np.testing.assert_array_equal(tgt[f][k], want[f][k])
    for k in "rgb":
        np.testing.assert_allclose(tgt["color"][k], want["color"][k], rtol=1e-5, atol=1e-5)
    tail = np.zeros(n, DATOS_MLP)
    orc.cpu.orc_tail(orc.p(regs), orc.p(tail), n)
    np.testing.assert_array_equal(tail.view(np.uint8), g["tail_out"])

    nd, batch = int(g["nd"]), int(g["batch"])
    idx = np.zeros(batch, np.int32)
    orc.cpu.orc_indices(orc.p(idx), nd, batch, 12345)
    np.testing.assert_array_equal(idx, g["indices"])
    datos = g["datos"].view(DATOS_MLP)
    bounds = np.ascontiguousarray(g["bounds"]).view(BOUNDS)
    tin, ttg = np.zeros(batch * 15, np.float32), np.zeros(batch * 3, np.float32)
    orc.cpu.orc_train_rows(orc.p(datos), orc.p(idx), batch, 15, 3, bounds.ctypes.data, orc.p(tin), orc.p(ttg))
    np.testing.assert_array_equal(tin.view(np.uint32), g["train_in"].view(np.uint32))
    # targets pass NaN through: same positions, payload bits may differ
    # (the device writes its canonical NaN)
    np.testing.assert_array_equal(ttg, g["train_tgt"])
    rows = np.zeros(nd * 15, np.float32)
    orc.cpu.orc_infer_rows(orc.p(datos), nd, 15, orc.p(rows), bounds.ctypes.data)
    np.testing.assert_array_equal(rows.view(np.uint32), g["infer_rows"].view(np.uint32))
    sc = np.zeros(nd, COLOR)
    orc.cpu.orc_scrub(orc.p(g["net"]), orc.p(sc), nd)
    np.testing.assert_array_equal(sc.view(np.uint8), g["scrub"])

    for (w, h) in ((512, 512), (1920, 1080), (7, 3)):
        c = np.zeros(1, CAMARA)
        orc.cpu.orc_default_camera(orc.p(c), w, h)
        want = g[f"camera_{w}x{h}"].view(CAMARA)
        for f in ("posicion", "frente", "arriba", "izquierda"):
            for k in "xyz":
                assert c[f][k] == want[f][k]
        assert abs(float(c["alto_plano"][0]) - float(want["alto_plano"][0])) <= 1e-6
