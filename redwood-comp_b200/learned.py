"""Training and evaluation of the boundary MLP of the learned-CDF sort.

Training data come from the pipeline itself: Gaussian-mixture clouds from
held-out seeds are Morton-encoded and sorted on the GPU (rw_tree_run_stage1/2),
the learned sort's own sampling code extracts the MLP inputs of every boundary
(rw_tree_learned_features), and the target of boundary j is where the true
quantile of rank (j+1) n / 4096 falls inside its window of sample keys.  The
network (16 -> 64 -> 64 -> 1, BF16 weights, FP32 master copy) is trained with
the project's own forward/backward and Adam kernels.

    python redwood-comp_b200/learned.py --out <table.json>
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PARAMS_PATH = os.path.join(HERE, "tuning", "cdf_mlp_b200.json")
N_PARAMS = 5313
N_BUCKETS = 4096

# seed ranges: training and evaluation never share a seed
TRAIN_SEED0, EVAL_SEED0 = 500_000, 900_000


def mixture_cloud(rw, n: int, seed: int):
    """A Gaussian mixture with 8-64 components (by seed), sigma 4-40."""
    k = 8 + (seed * 2654435761 % 57)
    return rw.generate_points(n, rw.GEN_GAUSSIAN_MIXTURE, seed, n_components=int(k),
                              sigma_lo=4.0, sigma_hi=40.0)


def morton_keys(rw, pts, sorted_too: bool = True):
    """(keys, sorted keys) of a cloud as device int32 tensors, made by the
    pipeline's stages 1 and 2."""
    n = pts.shape[0]
    app = rw.AppData(n, 32, points=pts)
    im = rw.ImStorage(n, 32)
    rw.run_stage1(app, im)
    if sorted_too:
        rw.run_stage2(app, im)
    return app.u_morton_keys, app.u_morton_keys_alt


def training_examples(rw, learned, seeds, n: int):
    """MLP inputs and targets of every boundary of every training cloud.

    The target of boundary j is where, inside its window [lo, hi] of sample
    keys, the full data's mass splits in half: the key of population rank
    (R(lo) + R(hi)) / 2 with R the rank among all keys, normalised to the
    window.  (Where the window lies is set by the sample; only how the mass is
    spread inside it can be learned.)"""
    import torch
    xs, ts = [], []
    for s in seeds:
        keys, srt = morton_keys(rw, mixture_cloud(rw, n, s))
        f, lo, span, _ = learned.features(keys)
        lo_t = torch.from_numpy(lo.view(np.int32)).to(srt.device)
        hi_t = torch.from_numpy((lo + span).view(np.int32)).to(srt.device)
        r_lo = torch.searchsorted(srt, lo_t, right=False)
        r_hi = torch.searchsorted(srt, hi_t, right=True)
        mid = torch.clamp((r_lo + r_hi) // 2, max=n - 1)
        key_mid = srt[mid].cpu().numpy().view(np.uint32).astype(np.float64)
        t = (key_mid - lo.astype(np.float64)) / span.astype(np.float64)
        xs.append(f)
        ts.append(np.clip(t, 0.0, 1.0).astype(np.float32))
    return np.concatenate(xs), np.concatenate(ts)


def init_params(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0, np.sqrt(2.0 / 16), (64, 16))
    w2 = rng.normal(0, np.sqrt(2.0 / 64), (64, 64))
    w3 = rng.normal(0, np.sqrt(1.0 / 64), 64)
    return np.concatenate([w1.ravel(), np.zeros(64), w2.ravel(), np.zeros(64), w3,
                           [0.5]]).astype(np.float32)


def train(rw, x: np.ndarray, t: np.ndarray, steps: int = 3000, batch: int = 8192,
          lr: float = 1e-3, seed: int = 0, log=print) -> tuple[np.ndarray, list]:
    import torch
    dev = torch.device("cuda")
    X = torch.from_numpy(x).to(dev)
    T = torch.from_numpy(t).to(dev)
    p = torch.from_numpy(init_params(seed)).to(dev)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    g = torch.zeros_like(p)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    hist = []
    for step in range(1, steps + 1):
        idx = torch.randint(0, X.shape[0], (batch,), device=dev, generator=gen)
        xb, tb = X[idx].contiguous(), T[idx].contiguous()
        g.zero_()
        loss.zero_()
        rw.mlp_grad(p, xb, tb, batch, g, loss)
        cur_lr = lr * 0.5 * (1 + np.cos(np.pi * step / steps))  # cosine decay
        rw.mlp_adam(p, g, m, v, float(cur_lr), step)
        if step % 500 == 0 or step == 1:
            hist.append((step, float(loss.item()) / batch))
            log(f"step {step}: mse {hist[-1][1]:.5f}")
    return p.cpu().numpy(), hist


def balance(counts: np.ndarray) -> dict:
    """Bucket balance: fullest bucket and spread relative to the mean."""
    c = counts.astype(np.float64)
    mean = c.mean()
    return {"max_over_mean": float(c.max() / mean), "cv": float(c.std() / mean),
            "max": int(c.max())}


def evaluate(rw, learned, seeds, n: int) -> dict:
    out = {"mlp": [], "sample_quantiles": []}
    for s in seeds:
        keys, _ = morton_keys(rw, mixture_cloud(rw, n, s), sorted_too=False)
        for mode, name in ((rw.LEARNED_MLP, "mlp"), (rw.LEARNED_SAMPLE_QUANTILES,
                                                      "sample_quantiles")):
            out[name].append(balance(learned.bucket_counts(keys, mode)))
    summary = {}
    for name, rows in out.items():
        summary[name] = {k: float(np.mean([r[k] for r in rows])) for k in rows[0]}
    return summary


def save_params(path: str, params: np.ndarray, meta: dict) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump({"params": [float(v) for v in params], **meta}, f)


def load_params(path: str = PARAMS_PATH):
    try:
        with open(path) as f:
            d = json.load(f)
        p = np.asarray(d["params"], np.float32)
        return p if p.size == N_PARAMS else None
    except (OSError, ValueError, KeyError):
        return None


def main(argv=None) -> int:
    import argparse
    sys.path.insert(0, os.path.dirname(HERE))
    from __graft_entry__ import _load_package
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", type=int, default=160)
    ap.add_argument("--eval-seeds", type=int, default=16)
    ap.add_argument("--n", type=int, default=8 << 20)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--out", default=PARAMS_PATH)
    a = ap.parse_args(argv)
    rw = _load_package()
    learned = rw.Learned(a.n, params=None)
    t0 = time.time()
    x, t = training_examples(rw, learned, range(TRAIN_SEED0, TRAIN_SEED0 + a.train_seeds), a.n)
    t1 = time.time()
    params, hist = train(rw, x, t, steps=a.steps)
    t2 = time.time()
    learned.set_params(params)
    ev = evaluate(rw, learned, range(EVAL_SEED0, EVAL_SEED0 + a.eval_seeds), a.n)
    meta = {"examples": int(x.shape[0]), "train_seeds": [TRAIN_SEED0, TRAIN_SEED0 + a.train_seeds],
            "eval_seeds": [EVAL_SEED0, EVAL_SEED0 + a.eval_seeds], "n_points": a.n,
            "steps": a.steps, "loss_history": hist, "eval": ev,
            "seconds": {"data": round(t1 - t0, 2), "train": round(t2 - t1, 2)}}
    save_params(a.out, params, meta)
    print(json.dumps({k: v for k, v in meta.items() if k != "loss_history"}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
