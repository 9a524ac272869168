"""Training and evaluation of the boundary MLP of the learned-CDF sort.

Training data come from the pipeline itself: Gaussian-mixture clouds from
held-out seeds are Morton-encoded and sorted on the GPU (rw_tree_run_stage1/2),
and the learned sort's own sampling code extracts the sorted 64K sample and
the MLP inputs of every boundary (rw_tree_learned_features).

Target.  A sample key's population rank R(s_i) is noisy: consecutive sample
keys are separated by exponentially distributed population masses, so the
plain sample quantile s_c (one order statistic per boundary) leaves every
bucket with the mass of 16 such gaps (coefficient of variation 1/4).  The
target of boundary j averages that noise over its whole context of 16g sample
keys: every context key s_i votes for the population rank R(s_i) + (c - i) n/m
as the rank of the boundary and the target rank rho is the mean vote.  The
network predicts where rho falls among the sample keys, as a fractional
sample rank relative to c divided by the context half-width 8g; the kernel
interpolates the boundary key between the two sample keys around it.  The
network sees only the sample keys' positions: it learns a smoothed inversion
of the sample's CDF (in regions of uniform density the answer is a linear
function of its inputs).

The network (16 -> 64 -> 64 -> 1, BF16 weights, FP32 master copy) is trained
with the project's own forward/backward and Adam kernels; the context group
size g is chosen on held-out evaluation seeds.

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
N_SAMPLE = 65536
SPACING = N_SAMPLE // N_BUCKETS

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


def context_rows(group: int):
    """(boundary indices whose context fits inside the sample, their sample
    ranks c, context half-width)."""
    j = np.arange(N_BUCKETS - 1)
    c = (j + 1) * SPACING
    half = (16 // 2) * group
    ok = (c >= half) & (c + half <= N_SAMPLE)
    return j[ok], c[ok], half


def interpolate(sample: np.ndarray, c: np.ndarray, half: int, y: np.ndarray) -> np.ndarray:
    """Boundary keys from network outputs y (as the kernel does, in float64)."""
    d = np.clip(y.astype(np.float64) * half, -half, half - 1)
    fl = np.floor(d)
    i0 = (c + fl).astype(np.int64)
    i1 = np.minimum(i0 + 1, N_SAMPLE - 1)
    a0 = sample[i0].astype(np.int64)
    gap = sample[i1].astype(np.int64) - a0
    return a0 + np.minimum(np.floor((d - fl) * gap + 0.5).astype(np.int64), gap)


def targets(srt, sample: np.ndarray, group: int):
    """Targets of the boundaries whose context fits (see the module doc).

    srt: the sorted population (device int32 tensor), sample: the sorted
    sample (uint32).  Returns (rows, targets, ideal boundary keys for all 4,095
    boundaries: the targets turned into keys as the kernel turns outputs into
    keys, the sample quantile where the context does not fit, then made
    non-decreasing)."""
    import torch
    n, m = srt.numel(), N_SAMPLE
    pop = srt.to(torch.int64) & 0xFFFFFFFF
    s = torch.from_numpy(sample.astype(np.int64)).to(srt.device)
    r = (torch.searchsorted(pop, s, right=False) + torch.searchsorted(pop, s, right=True))
    r = r.double().cpu().numpy() / 2.0          # population mid-rank of each sample key
    d = r - np.arange(m) * (n / m)              # each key's vote minus the ideal rank
    cs = np.concatenate([[0.0], np.cumsum(d)])
    rows, c, half = context_rows(group)
    rho = c * (n / m) + (cs[c + half] - cs[c - half]) / (2 * half)
    # fractional sample rank of rho (r is non-decreasing)
    i = np.clip(np.searchsorted(r, rho, side="right") - 1, 0, m - 2)
    den = r[i + 1] - r[i]
    frac = np.where(den > 0, np.clip((rho - r[i]) / np.where(den > 0, den, 1), 0, 1), 0.0)
    t = np.clip((i + frac - c) / half, -1.0, 1.0 - 1.0 / half)
    ideal = sample[(np.arange(N_BUCKETS - 1) + 1) * SPACING].astype(np.int64)
    ideal[rows] = interpolate(sample, c, half, t)
    return rows, t.astype(np.float32), np.maximum.accumulate(ideal).astype(np.uint32)


def counts_of(srt, bounds: np.ndarray) -> np.ndarray:
    """Keys per bucket when bucket(k) = number of boundaries <= k."""
    import torch
    pop = srt.to(torch.int64) & 0xFFFFFFFF
    b = torch.from_numpy(bounds.astype(np.int64)).to(srt.device)
    p = torch.searchsorted(pop, b, right=False).cpu().numpy()
    return np.diff(np.concatenate([[0], p, [srt.numel()]]))


def training_examples(rw, learned, seeds, n: int, groups):
    """{group: (inputs, targets)} over the clouds of `seeds`."""
    out = {g: ([], []) for g in groups}
    for s in seeds:
        keys, srt = morton_keys(rw, mixture_cloud(rw, n, s))
        for g in groups:
            learned.set_group(g)
            f, sample = learned.features(keys)
            rows, t, _ = targets(srt, sample, g)
            out[g][0].append(f[rows])
            out[g][1].append(t)
    return {g: (np.concatenate(x), np.concatenate(t)) for g, (x, t) in out.items()}


def init_params(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0, np.sqrt(2.0 / 16), (64, 16))
    w2 = rng.normal(0, np.sqrt(2.0 / 64), (64, 64))
    w3 = rng.normal(0, np.sqrt(1.0 / 64), 64)
    return np.concatenate([w1.ravel(), np.zeros(64), w2.ravel(), np.zeros(64), w3,
                           [0.0]]).astype(np.float32)


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


def evaluate(rw, learned, seeds, n: int, with_ideal: bool = False) -> dict:
    """Mean bucket balance over `seeds`: the network's boundaries, the plain
    sample quantiles and (with_ideal) the training targets themselves."""
    names = ["mlp", "sample_quantiles"] + (["ideal_targets"] if with_ideal else [])
    out = {k: [] for k in names}
    for s in seeds:
        keys, srt = morton_keys(rw, mixture_cloud(rw, n, s), sorted_too=with_ideal)
        out["mlp"].append(balance(learned.bucket_counts(keys, rw.LEARNED_MLP)))
        out["sample_quantiles"].append(
            balance(learned.bucket_counts(keys, rw.LEARNED_SAMPLE_QUANTILES)))
        if with_ideal:
            _, sample = learned.features(keys)
            out["ideal_targets"].append(balance(counts_of(srt, targets(srt, sample,
                                                                       learned.group)[2])))
    return {k: {q: float(np.mean([r[q] for r in rows])) for q in rows[0]}
            for k, rows in out.items()}


def save_params(path: str, params: np.ndarray, group: int, meta: dict) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump({"params": [float(v) for v in params], "group": int(group), **meta}, f)


def load_params(path: str = PARAMS_PATH, with_group: bool = False):
    """The trained parameters (or None); with_group: (params, group)."""
    p, g = None, 4
    try:
        with open(path) as f:
            d = json.load(f)
        q = np.asarray(d["params"], np.float32)
        if q.size == N_PARAMS:
            p, g = q, int(d.get("group", 4))
    except (OSError, ValueError, KeyError):
        pass
    return (p, g) if with_group else p


def main(argv=None) -> int:
    import argparse
    sys.path.insert(0, os.path.dirname(HERE))
    from __graft_entry__ import _load_package
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", type=int, default=160)
    ap.add_argument("--eval-seeds", type=int, default=16)
    ap.add_argument("--n", type=int, default=8 << 20)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--groups", default="2,4,8,16")
    ap.add_argument("--out", default=PARAMS_PATH)
    a = ap.parse_args(argv)
    groups = [int(v) for v in a.groups.split(",")]
    rw = _load_package()
    learned = rw.Learned(a.n, params=None)
    t0 = time.time()
    data = training_examples(rw, learned, range(TRAIN_SEED0, TRAIN_SEED0 + a.train_seeds),
                             a.n, groups)
    t1 = time.time()
    eval_seeds = range(EVAL_SEED0, EVAL_SEED0 + a.eval_seeds)
    results = {}
    for g in groups:
        x, t = data[g]
        params, hist = train(rw, x, t, steps=a.steps)
        learned.set_params(params, g)
        ev = evaluate(rw, learned, eval_seeds, a.n, with_ideal=True)
        results[g] = (params, hist, ev, int(x.shape[0]))
        print(json.dumps({"group": g, "examples": int(x.shape[0]), "eval": ev}), flush=True)
    best = min(groups, key=lambda g: results[g][2]["mlp"]["max_over_mean"])
    params, hist, ev, n_ex = results[best]
    meta = {"examples": n_ex, "train_seeds": [TRAIN_SEED0, TRAIN_SEED0 + a.train_seeds],
            "eval_seeds": [EVAL_SEED0, EVAL_SEED0 + a.eval_seeds], "n_points": a.n,
            "steps": a.steps, "loss_history": hist, "eval": ev,
            "sweep": {str(g): results[g][2] for g in groups},
            "seconds": {"data": round(t1 - t0, 2), "total": round(time.time() - t0, 2)}}
    save_params(a.out, params, best, meta)
    print(json.dumps({"chosen_group": best, "eval": ev}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
