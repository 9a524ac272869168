"""Test infrastructure: CPU (numpy, float32) restatement of the boundary MLP of
the learned-CDF sort, forward and backward, to check the GPU training kernels'
gradients, and the tensor-core inference numerics (forward_inference).
Weights are rounded to BF16 (round to nearest, ties to even) before use, as
the kernels do; in training the biases and all arithmetic stay float32.

Layout of the parameter vector: W1 [64][16], b1 [64], W2 [64][64], b2 [64],
W3 [64], b3 [1].
"""
import numpy as np

IN, H = 16, 64
SIZES = [("w1", H * IN), ("b1", H), ("w2", H * H), ("b2", H), ("w3", H), ("b3", 1)]
N_PARAMS = sum(s for _, s in SIZES)


def bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even) -> float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    r = ((u + rounding) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, size in SIZES:
        out[name] = p[o:o + size]
        o += size
    out["w1"] = out["w1"].reshape(H, IN)
    out["w2"] = out["w2"].reshape(H, H)
    return out


def forward(p: np.ndarray, x: np.ndarray) -> np.ndarray:
    q = unpack(np.asarray(p, np.float32))
    w1, w2, w3 = bf16_round(q["w1"]), bf16_round(q["w2"]), bf16_round(q["w3"])
    h1 = np.maximum(x @ w1.T + q["b1"], 0).astype(np.float32)
    h2 = np.maximum(h1 @ w2.T + q["b2"], 0).astype(np.float32)
    return (h2 @ w3 + q["b3"][0]).astype(np.float32)


def forward_inference(p: np.ndarray, x: np.ndarray) -> np.ndarray:
    """The inference numerics of the tensor-core kernels: inputs, W1, W2 and
    the hidden activations of layer 1 rounded to BF16, the two hidden layers'
    products summed exactly (float64, then float32) before the float32 bias,
    ReLU; the output b3 + sum_u w3[u] h2[u] in float32, units in order."""
    q = unpack(np.asarray(p, np.float32))
    w1, w2, w3 = bf16_round(q["w1"]), bf16_round(q["w2"]), bf16_round(q["w3"])
    xb = bf16_round(np.asarray(x, np.float32)).astype(np.float64)
    z1 = (xb @ w1.T.astype(np.float64)).astype(np.float32) + q["b1"]
    h1 = bf16_round(np.maximum(z1, 0).astype(np.float32)).astype(np.float64)
    z2 = (h1 @ w2.T.astype(np.float64)).astype(np.float32) + q["b2"]
    h2 = np.maximum(z2, 0).astype(np.float32)
    y = np.full(len(xb), q["b3"][0], np.float32)
    for u in range(H):
        y = (y + w3[u] * h2[:, u]).astype(np.float32)
    return y


def grad(p: np.ndarray, x: np.ndarray, t: np.ndarray, batch: int):
    """(gradient of sum((y - t)^2) / batch, sum of squared errors)."""
    q = unpack(np.asarray(p, np.float32))
    x = np.asarray(x, np.float32)
    w1, w2, w3 = bf16_round(q["w1"]), bf16_round(q["w2"]), bf16_round(q["w3"])
    z1 = (x @ w1.T + q["b1"]).astype(np.float32)
    h1 = np.maximum(z1, 0)
    z2 = (h1 @ w2.T + q["b2"]).astype(np.float32)
    h2 = np.maximum(z2, 0)
    y = (h2 @ w3 + q["b3"][0]).astype(np.float32)
    e = y - t
    dy = (2.0 * e / batch).astype(np.float32)
    dz2 = (np.outer(dy, w3) * (z2 > 0)).astype(np.float32)
    dh1 = dz2 @ w2
    dz1 = (dh1 * (z1 > 0)).astype(np.float32)
    g = {
        "w1": dz1.T @ x, "b1": dz1.sum(0), "w2": dz2.T @ h1, "b2": dz2.sum(0),
        "w3": h2.T @ dy, "b3": np.array([dy.sum()], np.float32),
    }
    flat = np.concatenate([np.asarray(g[name], np.float32).reshape(-1) for name, _ in SIZES])
    return flat, float((e * e).sum())
