"""CPU checks of the oracle's number-format helpers: its BF16 and E4M3
rounding must agree with torch's own conversions (an independent
implementation) before they are used to check the BF16 / FP8 kernels."""
import numpy as np
import torch

from oracle import mlp_oracle as mo


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(1).normal(size=20000).astype(np.float32) * np.float32(37.0)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(mo.round_bf16(x), want)


def test_e4m3_rounding_matches_torch_and_saturates():
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.normal(size=20000) * 40.0, rng.uniform(-0.02, 0.02, 2000), [448.0, -448.0, 0.0]])
    want = torch.from_numpy(np.clip(x, -448.0, 448.0)).to(torch.float8_e4m3fn).to(torch.float64).numpy()
    np.testing.assert_array_equal(mo.round_e4m3(x), want)
    assert mo.round_e4m3(np.array([1e6, -1e6])).tolist() == [448.0, -448.0]
    assert len(mo._E4M3) == 127   # 0, 7 subnormals, 119 normals


def test_quantized_forward_is_close_to_fp64():
    rng = np.random.default_rng(3)
    W = [rng.normal(0, 0.15, s) for s in mo.SHAPES]
    x = rng.uniform(-1, 1, (256, 96))
    ref = mo.forward(W, x)[0]
    scale = np.abs(ref).mean()
    bf = mo.forward_quantized(W, x, "bf16")
    f8 = mo.forward_quantized(W, x, "fp8", mo.layer_input_amax(W, x))
    # random 6-layer network: BF16 stays within ~1 %, E4M3 (3 mantissa bits)
    # within a few tens of percent of the mean output
    assert np.abs(bf - ref).mean() / scale < 0.02
    assert np.abs(f8 - ref).mean() / scale < 0.3
