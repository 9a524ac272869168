"""The boundary network's CPU oracle (oracle/mlp_oracle.py), on the CPU: its
BF16 rounding equals torch's float32 -> bfloat16 conversion (round to nearest
even), and the tensor-core inference numerics stay within BF16 precision of
the FP32-activation forward the network was trained with."""
import numpy as np

import mlp_oracle


def test_bf16_round_equals_torch():
    import torch
    rng = np.random.default_rng(5)
    x = np.concatenate([
        rng.normal(0, 1, 20000).astype(np.float32),
        rng.normal(0, 1e-3, 2000).astype(np.float32),
        rng.normal(0, 1e4, 2000).astype(np.float32),
        # exact ties between two BF16 values (low 16 bits 0x8000)
        (np.arange(2000, dtype=np.uint32) << 16 | 0x8000).view(np.float32),
    ])
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(mlp_oracle.bf16_round(x), want)


def test_inference_numerics_close_to_training_forward():
    rng = np.random.default_rng(6)
    p = rng.normal(0, 0.3, mlp_oracle.N_PARAMS).astype(np.float32)
    x = rng.random((500, mlp_oracle.IN), dtype=np.float32)
    a = mlp_oracle.forward(p, x)
    b = mlp_oracle.forward_inference(p, x)
    scale = float(np.abs(a).max())
    assert np.abs(a - b).max() <= 2e-2 * scale
    assert not np.array_equal(a, b)  # the activations really are rounded
