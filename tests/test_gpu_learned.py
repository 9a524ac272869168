"""Learned-CDF bucketed sort: the training kernels' gradients equal the CPU
oracle's, the sort's output equals the plain sort's on every input (MLP
boundaries, sample-quantile boundaries, the large-bucket path and the onesweep
fallback), and the trained network's effect on bucket balance is measured."""
import numpy as np
import pytest

import mlp_oracle

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def test_mlp_forward_and_grad_match_cpu_oracle(rw):
    torch = _torch()
    from redwood_comp_b200 import learned
    rng = np.random.default_rng(3)
    p = learned.init_params(7)
    p += rng.normal(0, 0.05, p.size).astype(np.float32)  # nonzero biases too
    rows = 1000
    x = rng.random((rows, 16), dtype=np.float32)
    t = rng.random(rows, dtype=np.float32)
    dp, dx, dt = (torch.from_numpy(a).cuda() for a in (p, x, t))
    y = rw.mlp_forward(dp, dx).cpu().numpy()
    want_y = mlp_oracle.forward_inference(p, x)
    # the tensor cores sum the products in FP32 in their own order; a hidden
    # value that lands next to a BF16 rounding midpoint may round the other
    # way (one BF16 step, 2^-8 relative), so a few rows move by ~1e-4
    err = np.abs(y - want_y)
    assert np.median(err) <= 2e-6 * max(1.0, float(np.abs(want_y).max())), np.median(err)
    np.testing.assert_allclose(y, want_y, rtol=2e-3, atol=2e-3)
    # and the network is the training network: FP32 activations agree to the
    # precision of BF16 activations
    np.testing.assert_allclose(y, mlp_oracle.forward(p, x), rtol=1e-2, atol=1e-2)
    g, loss = rw.mlp_grad(dp, dx, dt, rows)
    want, want_loss = mlp_oracle.grad(p, x, t, rows)
    # float32 sums in a different order: relative 1e-4 of the largest entry
    np.testing.assert_allclose(g.cpu().numpy(), want, rtol=1e-4,
                               atol=1e-4 * float(np.abs(want).max()))
    assert abs(float(loss.item()) - want_loss) <= 1e-4 * want_loss


def test_adam_step_matches_formula(rw):
    torch = _torch()
    rng = np.random.default_rng(4)
    p = rng.normal(0, 1, rw.MLP_PARAMS).astype(np.float32)
    g = rng.normal(0, 1, rw.MLP_PARAMS).astype(np.float32)
    dp, dg = torch.from_numpy(p.copy()).cuda(), torch.from_numpy(g).cuda()
    m, v = torch.zeros_like(dp), torch.zeros_like(dp)
    rw.mlp_adam(dp, dg, m, v, 1e-3, 1)
    mm, vv = 0.1 * g, 0.001 * g * g
    want = p - 1e-3 * (mm / 0.1) / (np.sqrt(vv / 0.001) + 1e-8)
    np.testing.assert_allclose(dp.cpu().numpy(), want, rtol=1e-5, atol=1e-6)


def _keys(rw, n, kind, seed):
    torch = _torch()
    from redwood_comp_b200 import learned
    if kind == "gauss":
        pts = learned.mixture_cloud(rw, n, seed)
    else:
        pts = rw.generate_points(n, rw.GEN_UNIFORM, seed)
    keys, _ = learned.morton_keys(rw, pts, sorted_too=False)
    return keys.clone()


@pytest.mark.parametrize("n", [65536, 1_000_003, 16_777_216])
def test_learned_sort_equals_plain_sort(rw, n):
    torch = _torch()
    from redwood_comp_b200 import learned
    L = rw.Learned(n)  # the trained table and its group size, when present
    if L.params is None:
        L.set_params(learned.init_params(1))
    im = rw.ImStorage(n, 32)
    for kind in ("gauss", "uniform"):
        keys = _keys(rw, n, kind, 41 + n % 97)
        want = np.sort(keys.cpu().numpy().view(np.uint32))
        for mode in (rw.LEARNED_MLP, rw.LEARNED_SAMPLE_QUANTILES):
            out, st = L.sort(keys, mode=mode, fallback_im=im)
            got = out.cpu().numpy().view(np.uint32)
            assert np.array_equal(got, want), (n, kind, mode, st)
            assert st["fell_back"] == 0


def test_learned_sort_large_bucket_and_fallback(rw):
    """A bucket above one CTA's capacity takes the chunked path; a bucket above
    its region (4x the mean bucket size) sends everything to onesweep."""
    torch = _torch()
    n = 1 << 26  # mean bucket 16,384 keys, region 65,536
    L = rw.Learned(n, params=None)
    im = rw.ImStorage(n, 32)
    rng = np.random.default_rng(9)
    k = rng.integers(0, 1 << 30, n, dtype=np.uint64).astype(np.uint32)
    k[rng.choice(n, 40_000, replace=False)] = 123456789  # one bucket of ~56K keys
    keys = torch.from_numpy(k.view(np.int32)).cuda()
    out, st = L.sort(keys, mode=rw.LEARNED_SAMPLE_QUANTILES, fallback_im=im)
    assert st["big_buckets"] >= 1 and st["fell_back"] == 0, st
    assert np.array_equal(out.cpu().numpy().view(np.uint32), np.sort(k))
    del keys, out
    # every key equal: one bucket with everything overflows -> onesweep
    m = 4 << 20
    same = torch.full((m,), 77, dtype=torch.int32, device="cuda")
    out, st = L.sort(same, mode=rw.LEARNED_SAMPLE_QUANTILES, fallback_im=im)
    assert st["fell_back"] == 1
    assert bool((out == 77).all())


def test_bucket_counts_fit_regions(rw):
    """Trained boundaries on held-out mixtures: counts add up to n and no
    bucket comes near its region."""
    from redwood_comp_b200 import learned
    n = 1 << 24
    L = rw.Learned(n)
    cap = 4 * (n // 4096)
    for seed in (910_001, 910_002):
        keys = _keys(rw, n, "gauss", seed)
        for mode in (rw.LEARNED_MLP, rw.LEARNED_SAMPLE_QUANTILES):
            if mode == rw.LEARNED_MLP and L.params is None:
                continue
            c = L.bucket_counts(keys, mode)
            assert int(c.sum()) == n
            assert int(c.max()) < cap // 1.2, (seed, mode, int(c.max()))


@pytest.mark.parametrize("group", [1, 2, 16])
def test_learned_sort_exact_for_every_group(rw, group):
    """Untrained weights and every context width: boundaries stay monotone
    (the clamp), so the output is still exactly sorted."""
    from redwood_comp_b200 import learned
    n = 1_000_003
    L = rw.Learned(n, params=learned.init_params(5), group=group)
    im = rw.ImStorage(n, 32)
    keys = _keys(rw, n, "gauss", 77)
    out, st = L.sort(keys, mode=rw.LEARNED_MLP, fallback_im=im)
    assert np.array_equal(out.cpu().numpy().view(np.uint32),
                          np.sort(keys.cpu().numpy().view(np.uint32)))


@pytest.mark.parametrize("group", [1, 4, 16])
def test_features_match_numpy_restatement(rw, group):
    """The kernel's MLP inputs equal a float64 restatement from the sorted
    sample it returns: mean positions of eight groups of 2g context keys, then
    the positions of the keys of ranks c-4 .. c+3, normalised to the context."""
    from redwood_comp_b200 import learned
    n = 1 << 20
    L = rw.Learned(n, params=None, group=group)
    keys = _keys(rw, n, "gauss", 13)
    f, sample = L.features(keys)
    assert np.all(np.diff(sample.astype(np.int64)) >= 0)
    assert np.isin(sample, keys.cpu().numpy().view(np.uint32)).all()
    rows, c, half = learned.context_rows(group)
    s = sample.astype(np.float64)
    lo = s[c - half]
    span = np.maximum(s[c + half - 1] - lo, 1.0)
    ctx = np.stack([s[c - half + i] for i in range(2 * half)], 1) - lo[:, None]
    coarse = ctx.reshape(len(rows), 8, 2 * group).mean(2) / span[:, None]
    fine = (np.stack([s[c - 4 + i] for i in range(8)], 1) - lo[:, None]) / span[:, None]
    np.testing.assert_allclose(f[rows], np.concatenate([coarse, fine], 1), rtol=4e-7, atol=1e-7)
    others = np.setdiff1d(np.arange(4095), rows)
    assert np.all(f[others] == 0)


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("mode", [0, 1])
def test_pipeline_with_learned_sort_matches_oracle(rw, oracle, fused, mode):
    """Stage 2 by the learned sort (set on the pipeline's scratch): all seven
    stages stay bit-exact against the oracle, fused and stage by stage."""
    from redwood_comp_b200 import learned
    from test_gpu_parity import run_gpu, assert_same
    n = 1_000_003
    pts = learned.mixture_cloud(rw, n, 20_017)
    L = rw.Learned(n)
    if L.params is None:
        L.set_params(learned.init_params(1))
    im = rw.ImStorage(n, 32)
    im.set_learned(L, mode)
    got = run_gpu(rw, pts, fused=fused, im=im)
    assert im.learned_stats()["fell_back"] == 0
    assert_same(got, oracle.run(pts, key_bits=32), f"learned mode {mode} fused {fused}")
    # back to onesweep on the same scratch
    im.set_learned(None)
    assert_same(run_gpu(rw, pts, fused=fused, im=im), oracle.run(pts, key_bits=32), "onesweep")


def test_trained_network_gains_over_sample_quantiles(rw):
    """What the trained boundary MLP buys over the method without it (plain
    sample quantiles of the same 64K-key sample): on held-out mixtures (seeds
    the network never saw) its buckets are more even, both in spread (cv) and
    in the fullest bucket.  (Sort speed is a separate matter: both sorts run
    the same kernels, and bench.py reports their times.)"""
    from redwood_comp_b200 import learned
    L = rw.Learned(1 << 23)
    if L.params is None:
        pytest.skip("no trained table")
    n = 1 << 23
    mlp, sq = [], []
    for seed in range(learned.EVAL_SEED0 + 100, learned.EVAL_SEED0 + 106):
        keys, _ = learned.morton_keys(rw, learned.mixture_cloud(rw, n, seed), sorted_too=False)
        mlp.append(learned.balance(L.bucket_counts(keys, rw.LEARNED_MLP)))
        sq.append(learned.balance(L.bucket_counts(keys, rw.LEARNED_SAMPLE_QUANTILES)))
    cv_m = np.mean([b["cv"] for b in mlp]); cv_s = np.mean([b["cv"] for b in sq])
    mx_m = np.mean([b["max_over_mean"] for b in mlp])
    mx_s = np.mean([b["max_over_mean"] for b in sq])
    print(f"bucket cv: mlp {cv_m:.4f} vs sample quantiles {cv_s:.4f}; "
          f"max/mean: mlp {mx_m:.3f} vs {mx_s:.3f}")
    assert cv_m < 0.97 * cv_s
    assert mx_m < mx_s


def test_learned_pipeline_replayed_from_a_cuda_graph(rw, oracle):
    """With the learned sort in stage 2 the fused pipeline needs no host wait
    (the overflow fallback is decided on the device), so it captures into a
    CUDA graph; replays on clouds that take the bucket path and on one whose
    single dense spot overflows its bucket region (the gated onesweep sort
    runs instead) are all exact against the oracle."""
    import torch
    from redwood_comp_b200 import learned
    from test_gpu_parity import assert_same
    n = 1 << 20
    L = rw.Learned(n)
    if L.params is None:
        L.set_params(learned.init_params(1))
    app = rw.AppData(n, 32, points=learned.mixture_cloud(rw, n, 31_001))
    im = rw.ImStorage(n, 32)
    im.set_learned(L, rw.LEARNED_MLP)
    rw.run_pipeline(app, im)  # first run outside the capture
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        rw.pipeline_enqueue(app, im)
    dense = rw.generate_points(n, rw.GEN_UNIFORM, 31_004)
    dense[: n // 5] = np.float32(333.25)  # a fifth of the points on one spot
    for name, pts, fell_back in (("mixture", learned.mixture_cloud(rw, n, 31_002), 0),
                                 ("dense spot", dense, 1),
                                 ("mixture again", learned.mixture_cloud(rw, n, 31_003), 0)):
        app.set_points(pts)
        g.replay()
        rw.pipeline_finish(app, im)
        assert im.learned_stats()["fell_back"] == fell_back, name
        assert_same(app.results(), oracle.run(pts), f"graph replay {name}")
    del g
    im.set_learned(None)
