#!/usr/bin/env python
"""Benchmark of the B200 tree pipeline (7 stages, bit-exact): points/sec.

Default workload: the plain pipeline at scale, n = 16,777,216 points uniform
in [0, 1024)^3, 32-bit Morton keys, one cloud per GPU ("replicas only": the
path does not shard; with --gpus N every rank builds its own cloud's octree).

  value    - points/s with the points already in HBM: K back-to-back runs of
             the fused pipeline (rw_tree_pipeline_enqueue), CUDA events on the
             launching stream, max over ranks.
  e2e      - the same metric through rw_tree_run_host with pinned host
             buffers: H2D of the points, the pipeline, D2H of the counts and
             the octree rows, every step.
  roofline - the dominant kernel's algorithmic bytes per launch / its mean
             CUDA-event duration inside the pipeline, against the measured
             HBM copy bandwidth.
  cpu_baseline - the reference's own CPU path (cpu::run_stage1..7 compiled
             from its sources, oracle/_ref) on all host cores, rank 0, N = 1.

`--impl reference` times only the reference's CPU path on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "octree-build points/sec (7 stages, bit-exact): plain vs batched/learned, 1 B200"
# warp ranking schemes of the onesweep variants (rw_tree_sort_variant_info rank_mode)
RANK_NAMES = ("ballot", "match_any", "atomic_or", "half_packed", "atomic_or+ballot_top")
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--n", type=int, default=16777216)
    p.add_argument("--dist", choices=("uniform", "gauss", "appdata"), default="uniform")
    p.add_argument("--key-bits", type=int, default=32, choices=(32, 64))
    p.add_argument("--radix-bits", type=int, default=0, choices=(0, 8, 10, 11))
    p.add_argument("--seed", type=int, default=20260101)
    p.add_argument("--no-verify", action="store_true", help="skip the oracle check")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--sort-variant", type=int, default=-1,
                   help="onesweep variant index (default: the storage's default)")
    p.add_argument("--only-device", action="store_true",
                   help="time only the device-resident pipeline (for profiler runs)")
    p.add_argument("--slots", type=int, default=2,
                   help="clouds in flight in the device-resident timed region (AppData / "
                        "scratch pairs on their own streams, steps taken in turn)")
    p.add_argument("--e2e-slots", type=int, default=3,
                   help="AppData / scratch pairs and streams of the end-to-end region")
    p.add_argument("--no-forms", action="store_true",
                   help="skip the batched and learned forms in the default line")
    # internal: time the reference's CPU path in a child process (see ref_time_isolated)
    p.add_argument("--ref-time-child", action="store_true", help=argparse.SUPPRESS)
    # internal: time the reference's CUDA path in a child process (see ref_cuda_isolated)
    p.add_argument("--ref-cuda-child", action="store_true", help=argparse.SUPPRESS)
    p.add_argument("--no-ref-cuda", action="store_true",
                   help="skip timing the reference's own CUDA path")
    p.add_argument("--ref-threads", type=int, default=0, help=argparse.SUPPRESS)
    p.add_argument("--ref-iters", type=int, default=1, help=argparse.SUPPRESS)
    return p.parse_args()


def make_points(rw, n, dist, seed):
    """The workload's cloud from the library's generator (our arm)."""
    if dist == "appdata":
        return rw.generate_points(n, rw.GEN_APPDATA, 114514)
    if dist == "uniform":
        return rw.generate_points(n, rw.GEN_UNIFORM, seed)
    return rw.generate_points(n, rw.GEN_GAUSSIAN_MIXTURE, seed, n_components=32,
                              sigma_lo=4.0, sigma_hi=40.0)


def make_points_checker(n, dist, seed):
    """The same cloud without the product library (the reference arm and its
    timing child): the counter-based kinds from the oracle's C restatement of
    the generator, AppData's mt19937 stream from the reference's own code."""
    from oracle import Oracle, RefTree
    if dist == "appdata":
        return RefTree().default_points(n)
    if dist == "uniform":
        return Oracle().generate_points(n, 1, seed)
    return Oracle().generate_points(n, 2, seed, n_components=32, sigma_lo=4.0, sigma_hi=40.0)


def sort_passes(a):
    return -(-(30 if a.key_bits == 32 else 63) // (a.radix_bits or 8))


def config_of(a):
    """The `config` object of the JSON line; both arms print the same one."""
    return {"workload": workload_name(a), "n_points": a.n, "key_bits": a.key_bits,
            "radix_bits": a.radix_bits or 8, "sort_passes": sort_passes(a),
            "parallelism": f"replicas x{a.gpus} (one cloud per GPU)",
            "l2": f"inputs larger than L2 (points {16 * a.n / 1e6:.0f} MB per step)"
                  if 16 * a.n > (126 << 20) else "inputs smaller than L2"}


def workload_name(a):
    d = {"uniform": "uniform [0,1024)^3", "gauss": "32-component Gaussian mixture sigma 4-40",
         "appdata": "AppData mt19937(114514) uniform"}[a.dist]
    return f"plain tree pipeline (7 stages), n={a.n:,} points, {d}, {a.key_bits}-bit Morton"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region.

    NVML's read-only clock and clock-event-reason queries, from a thread, about
    every millisecond while the region runs, so that a region of a few
    milliseconds still has samples under load; the region starts after the
    first sample.  Without NVML: nvidia-smi every 200 ms around the region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    # NVML clock-event-reason bits (nvml.h nvmlClocksEventReason*)
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
                   ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, gpu_index, period_s=0.001):
        self.gpu = gpu_index
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.samples = []
        self.lines = []

    def _nvml_handle(self, nv):
        """The NVML device of this process's CUDA device: by PCI address when
        torch reports it (CUDA ordinals and NVML indices differ under
        CUDA_VISIBLE_DEVICES), else by index."""
        try:
            import torch
            pr = torch.cuda.get_device_properties(torch.cuda.current_device())
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus), "pci"
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.gpu), "index"

    def _loop(self):
        nv = self.nvml
        while True:
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                self.first.set()
                return
            self.samples.append((float(sm), int(rs)))
            self.first.set()
            if self.stop.wait(self.period):
                return

    def __enter__(self):
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            self.nvml = nv
            self.h, self.match = self._nvml_handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
            self.stop, self.first = threading.Event(), threading.Event()
            self.thread = threading.Thread(target=self._loop, daemon=True)
            self.thread.start()
            self.first.wait(1.0)
            return self
        except Exception:
            if self.nvml is not None:
                try:
                    self.nvml.nvmlShutdown()
                except Exception:
                    pass
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.nvml is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
            return False
        if self.proc is None:
            return False
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        self.lines = [ln for ln in out.splitlines() if ln.strip()]
        return False

    def summary(self):
        if self.samples:
            sm = [x for x, _ in self.samples]
            reasons = sorted({nm for _, rs in self.samples for nm, bit in self.REASON_BITS
                              if rs & bit})
            return {"sm_mhz": statistics.median(sm), "sm_min_mhz": min(sm),
                    "sm_max_mhz": self.max_mhz, "samples": len(sm), "reasons": reasons,
                    "source": f"nvml every {self.period * 1e3:g} ms inside the timed region "
                              f"(device by {self.match})"}
        if not self.lines:
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "samples": len(sm),
                "reasons": sorted(reasons), "source": "nvidia-smi every 200 ms around the region"}


def kernel_bytes(name, n, u, m, K):
    """Algorithmic bytes of one launch (each input read once, each output
    written once; neighbour reads counted as cache hits)."""
    b = max(u - 1, 0)
    if name == "morton_histogram":
        return (16 + K) * n
    if name.startswith("sort_pass"):
        return 2 * K * n
    if name == "unique":
        return K * n + K * u
    if name == "radix_tree_edges":
        # codes read; prefix_n, 2 leaf flags, left_child, parent, edge count written
        return K * u + 15 * b
    if name == "edge_scan":
        # counts read (per-tile sums; the offsets are written by the octree kernel)
        return 4 * b
    if name == "octree":
        # codes, prefix_n, count, parent read, offset written; corner 16 + cell 4
        # + children 32 + masks 8 written (links merged in shared memory)
        return (K + 13) * b + 60 * m
    return 0


def pipeline_bytes(n, u, m, K, passes):
    """Whole-pipeline algorithmic bytes (per-stage formulas: S1 (16+K)n,
    S2 K n (1+2P), S3 K(n+u), S4 K u + 11 b, S5 10 b, S6 4 b,
    S7 (13+K) b + 60 m; stage 6's offsets are written inside stage 7)."""
    b = u - 1
    return ((16 + K) * n + K * n * (1 + 2 * passes) + K * (n + u) + K * u + 11 * b
            + 10 * b + 4 * b + (13 + K) * b + 60 * m)


def traffic_table():
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def run_reference(a, rank):
    if rank != 0:
        return 0
    from oracle import ref_available
    pts = make_points_checker(a.n, a.dist, a.seed)
    note = None
    ms = None
    if a.key_bits == 32 and ref_available():
        ms, cores = ref_time_isolated(a, a.seed, a.warmup + a.steps)
        if ms is not None:
            kind = "reference"
            ms = ms[a.warmup:]
        else:
            note = cores
    if ms is None:
        # the reference has no 64-bit path (or failed on this cloud): the C
        # restatement stands in
        kind, cores = "port", 1
        port_time(pts, a, a.warmup)
        ms = port_time(pts, a, a.steps)
    t = statistics.median(ms)
    val = a.n / (t / 1e3)
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "points/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": t,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": f"u{a.key_bits}", "data": "synthetic",
        "config": config_of(a),
        "cpu_baseline": {"value": val, "unit": "points/s", "cores": cores, "kind": kind,
                         "sample": f"{a.steps} full runs of stages 1-7 on the n={a.n} cloud, "
                                   f"median wall time"},
        "e2e": {"value": val, "unit": "points/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if note:
        line["cpu_baseline"]["note"] = note
    print(json.dumps(line), flush=True)
    return 0


def batch_clouds(rw, n_clouds, seed, lo=1024, hi=262144):
    """The batched configuration: sizes log-uniform in [lo, hi], each cloud
    uniform or a Gaussian mixture with 8-64 components, chosen by seed."""
    rng = np.random.default_rng(seed)
    clouds = []
    for c in range(n_clouds):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        if rng.random() < 0.5:
            clouds.append(rw.generate_points(n, rw.GEN_UNIFORM, seed * 7919 + c))
        else:
            clouds.append(rw.generate_points(n, rw.GEN_GAUSSIAN_MIXTURE, seed * 7919 + c,
                                             n_components=int(rng.integers(8, 65))))
    return clouds


def measure_batch(rw, a, n_clouds=1024, verify_clouds=96):
    """Batched pipeline (one graph launch per run) against the plain pipeline
    run once per cloud on the same clouds, both bit-exact per cloud."""
    import torch
    from oracle import Oracle, ORC_OK
    clouds = batch_clouds(rw, n_clouds, a.seed + 3)
    total = int(sum(c.shape[0] for c in clouds))
    ratio = 1.0  # octree rows per point: room for every cloud (0.6 overflows small ones)
    batch = rw.Batch(clouds, a.key_bits, octree_ratio=ratio)
    for _ in range(max(3, a.warmup)):
        batch.run(graph=True)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(a.steps):
        batch.enqueue(graph=True)
    e1.record(s)
    batch.finish()
    batch_ms = e0.elapsed_time(e1) / a.steps
    failed = int((batch.status != 0).sum())

    # the plain pipeline once per cloud, launches back to back (no host sync
    # between clouds), same capacity ratio
    apps = [rw.AppData(c.shape[0], a.key_bits, points=c, octree_ratio=ratio) for c in clouds]
    im_big = rw.ImStorage(max(c.shape[0] for c in clouds), a.key_bits)

    def plain_once():
        for app in apps:
            rw.pipeline_enqueue(app, im_big)
        rw.pipeline_finish(apps[-1], im_big)

    plain_once()
    torch.cuda.synchronize()
    e0.record(s)
    reps = 2
    for _ in range(reps):
        plain_once()
    e1.record(s)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1) / reps

    mism = 0
    orc = Oracle()
    rng = np.random.default_rng(5)
    for c in sorted(rng.choice(n_clouds, size=min(verify_clouds, n_clouds), replace=False)):
        want = orc.run(clouds[c], key_bits=a.key_bits, capacity=batch.capacity(c))
        if want.status != ORC_OK:
            mism += int(batch.status[c] == 0)
            continue
        got, w = batch.results(int(c)), want.trimmed()
        mism += int(any(
            np.ascontiguousarray(got[k]).tobytes() != np.ascontiguousarray(v).tobytes()
            if isinstance(v, np.ndarray) else got[k] != v for k, v in w.items()))
    info = {
        "workload": f"batched: {n_clouds} clouds, sizes log-uniform in [1024, 262144] "
                    f"(total {total:,} points), uniform or 8-64 component Gaussian mixture by "
                    f"seed, {a.key_bits}-bit keys, octree rows {ratio} per point",
        "value": total / (batch_ms / 1e3), "unit": "points/s", "ms_per_batch": batch_ms,
        "plain_per_cloud_value": total / (plain_ms / 1e3), "plain_per_cloud_ms": plain_ms,
        "speedup_vs_plain": plain_ms / batch_ms,
        "clouds_failed": failed, "clouds_verified": min(verify_clouds, n_clouds),
        "mismatches_vs_oracle": mism,
        "tuning": batch.tuning and {"radix_bits": batch.tuning["radix_bits"],
                                    "classes": [(c["max_points"],
                                                 f'{c["threads"]}x{c["keys_per_thread"]} '
                                                 f'{RANK_NAMES[c["rank"]]}')
                                                for c in batch.tuning["classes"]]},
        "graph": True,
    }
    batch.close()
    return info


def measure_combined(rw, a, n_clouds=64, lo=1 << 20, hi=8 << 20, seed=880_001):
    """The combined configuration: 64 clouds, sizes log-uniform in [1M, 8M],
    Gaussian mixtures with 8-64 components, through the batched pipeline
    against the plain pipeline run once per cloud, every cloud's outputs
    compared on the device with its plain run.  64-bit keys with the batched
    onesweep sort; then the same clouds with 32-bit keys, the batched pipeline
    with the learned-CDF sort (MLP boundaries) as stage 2 of every cloud
    against the batched onesweep and the plain per-cloud runs (the learned
    sort serves 32-bit keys)."""
    import torch
    rng = np.random.default_rng(seed)
    sizes = [int(np.exp(rng.uniform(np.log(lo), np.log(hi)))) for _ in range(n_clouds)]
    clouds = [rw.generate_points(nc, rw.GEN_GAUSSIAN_MIXTURE, seed + c,
                                 n_components=int(8 + (seed + c) * 2654435761 % 57),
                                 sigma_lo=4.0, sigma_hi=40.0)
              for c, nc in enumerate(sizes)]
    total = int(sum(sizes))
    ratio = 1.0
    s = torch.cuda.current_stream()
    reps = 3

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def compare(batch, apps, im):
        mism = 0
        for c, app in enumerate(apps):  # every cloud against its own plain run
            rw.run_pipeline(app, im)
            p0 = int(batch.point_offsets[c])
            r0 = int(batch.octree_offsets[c])
            u, m = app.get_n_unique(), app.get_n_octree_nodes()
            same = int(batch.n_unique[c]) == u and int(batch.n_octree_nodes[c]) == m
            pairs = [(batch.morton_keys_alt[p0:p0 + app.n_input], app.u_morton_keys_alt),
                     (batch.morton_keys[p0:p0 + u], app.u_morton_keys[:u])]
            for bf, af in (("prefix_n", "brt_prefix_n"), ("has_leaf_left", "brt_has_leaf_left"),
                           ("has_leaf_right", "brt_has_leaf_right"),
                           ("left_child", "brt_left_child"), ("parents", "brt_parents"),
                           ("edge_count", "u_edge_count"), ("edge_offset", "u_edge_offset")):
                pairs.append((getattr(batch, bf)[p0:p0 + u - 1], getattr(app, af)[:u - 1]))
            for bf, af in (("children", "oct_children"), ("corner", "oct_corner"),
                           ("cell_size", "oct_cell_size"),
                           ("child_node_mask", "oct_child_node_mask"),
                           ("child_leaf_mask", "oct_child_leaf_mask")):
                pairs.append((getattr(batch, bf)[r0:r0 + m], getattr(app, af)[:m]))
            mism += int(not same or not all(torch.equal(x, y) for x, y in pairs))
        return mism

    def run_width(key_bits, learned_too):
        batch = rw.Batch(clouds, key_bits, octree_ratio=ratio)
        out = {}
        batch_ms = timed(lambda: batch.run(graph=True))
        failed = int((batch.status != 0).sum())
        im = rw.ImStorage(max(sizes), key_bits)
        apps = [rw.AppData(nc, key_bits, points=cl, octree_ratio=ratio)
                for nc, cl in zip(sizes, clouds)]

        def plain_once():
            for app in apps:
                rw.pipeline_enqueue(app, im)
            rw.pipeline_finish(apps[-1], im)

        plain_ms = timed(plain_once)
        out["onesweep"] = {"value": total / (batch_ms / 1e3), "ms_per_batch": batch_ms,
                           "speedup_vs_plain": plain_ms / batch_ms, "clouds_failed": failed,
                           "mismatched_clouds": compare(batch, apps, im)}
        if learned_too:
            L = rw.Learned(max(sizes))
            fb = rw.ImStorage(max(sizes), key_bits)
            if L.params is not None:
                batch.set_learned(L, rw.LEARNED_MLP, fb)
                lms = timed(lambda: batch.run(graph=True))
                out["learned_mlp"] = {
                    "value": total / (lms / 1e3), "ms_per_batch": lms,
                    "speedup_vs_plain": plain_ms / lms, "speedup_vs_batched_onesweep":
                        batch_ms / lms, "clouds_failed": int((batch.status != 0).sum()),
                    "mismatched_clouds": compare(batch, apps, im)}
                batch.set_learned(None)
            L.close()
        out["plain_per_cloud_value"] = total / (plain_ms / 1e3)
        out["plain_per_cloud_ms"] = plain_ms
        batch.close()
        del apps, im
        torch.cuda.empty_cache()
        return out

    w64 = run_width(64, False)
    w32 = run_width(32, True)
    info = {
        "workload": f"combined: {n_clouds} clouds, sizes log-uniform in [1M, 8M] (total "
                    f"{total:,} points), Gaussian mixtures with 8-64 components, octree rows "
                    f"{ratio} per point",
        "unit": "points/s", "graph": True,
        # the 64-bit line (BASELINE's key width for this configuration)
        "value": w64["onesweep"]["value"], "ms_per_batch": w64["onesweep"]["ms_per_batch"],
        "plain_per_cloud_value": w64["plain_per_cloud_value"],
        "plain_per_cloud_ms": w64["plain_per_cloud_ms"],
        "speedup_vs_plain": w64["onesweep"]["speedup_vs_plain"],
        "clouds_failed": w64["onesweep"]["clouds_failed"],
        "clouds_compared_with_plain": n_clouds,
        "mismatched_clouds": w64["onesweep"]["mismatched_clouds"],
        "key_bits_64": w64, "key_bits_32": w32,
    }
    return info


LEARNED_SEED = 950_001  # held out: the boundary MLP trains on seeds 500,000-500,159


def measure_learned(rw, a, n=67_108_864, reps=10):
    """Learned-CDF form: the full pipeline with the learned sort in stage 2
    against the plain pipeline, 67,108,864 points of a Gaussian mixture with
    8-64 components (32-bit keys), every output compared on the device."""
    import torch
    from redwood_comp_b200 import learned as lmod
    pts = lmod.mixture_cloud(rw, n, LEARNED_SEED)
    k_comp = 8 + (LEARNED_SEED * 2654435761 % 57)
    app_p = rw.AppData(n, 32, points=pts)
    app_l = rw.AppData(n, 32, points=pts)
    del pts
    im_p = rw.ImStorage(n, 32)
    im_l = rw.ImStorage(n, 32)
    L = rw.Learned(n)
    if L.params is None:
        return {"unavailable": "no trained boundary MLP table"}
    s = torch.cuda.current_stream()

    def timed(fn, k):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(k):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    plain_ms = timed(lambda: rw.pipeline_enqueue(app_p, im_p), reps)
    rw.pipeline_finish(app_p, im_p)
    out = {}
    for mode, name in ((rw.LEARNED_MLP, "mlp"), (rw.LEARNED_SAMPLE_QUANTILES, "sample_quantiles")):
        im_l.set_learned(L, mode)
        ms = timed(lambda: rw.pipeline_enqueue(app_l, im_l), reps)
        rw.pipeline_finish(app_l, im_l)
        same = app_l.get_n_unique() == app_p.get_n_unique() and \
            app_l.get_n_octree_nodes() == app_p.get_n_octree_nodes()
        mism = []
        for f in ("u_morton_keys_alt", "brt_prefix_n", "brt_has_leaf_left", "brt_has_leaf_right",
                  "brt_left_child", "brt_parents", "u_edge_count", "u_edge_offset",
                  "oct_children", "oct_corner", "oct_cell_size", "oct_child_node_mask",
                  "oct_child_leaf_mask"):
            x, y = getattr(app_l, f), getattr(app_p, f)
            if f.startswith("oct_"):
                x, y = x[:app_p.get_n_octree_nodes()], y[:app_p.get_n_octree_nodes()]
            elif not f.startswith("u_morton"):
                x, y = x[:app_p.get_n_unique()], y[:app_p.get_n_unique()]
            if not torch.equal(x, y):
                mism.append(f)
        out[name] = {"value": n / (ms / 1e3), "ms_per_step": ms,
                     "speedup_vs_plain": plain_ms / ms, "stats": im_l.learned_stats(),
                     "mismatched_outputs_vs_plain": mism if same else ["counts"] + mism}
    im_l.set_learned(None)
    # the sort alone, same keys
    keys = app_p.u_morton_keys.clone()
    sorted_out = torch.empty_like(keys)
    sort_ms = {"onesweep": timed(lambda: rw.sort_keys(keys, sorted_out, im_p), reps)}
    for mode, name in ((rw.LEARNED_MLP, "learned_mlp"),
                       (rw.LEARNED_SAMPLE_QUANTILES, "learned_sample_quantiles")):
        sort_ms[name] = timed(lambda: L.sort(keys, out=sorted_out, mode=mode, fallback_im=im_p),
                              reps)
    info = {
        "workload": f"learned-CDF: {n:,} points, Gaussian mixture with {k_comp} components "
                    f"(sigma 4-40, seed {LEARNED_SEED}, not a training seed), 32-bit keys",
        "plain_value": n / (plain_ms / 1e3), "plain_ms_per_step": plain_ms,
        "learned": out, "sort_only_ms": {k: round(v, 4) for k, v in sort_ms.items()},
        "boundary_mlp": {"group": L.group, "params": int(L.params.size)},
        "unit": "points/s",
    }
    L.close()
    return info


def ref_time_child(a):
    """Child side of ref_time_isolated: the same seeded cloud, the reference's
    verbatim stages 1-7 timed `--ref-iters` times; prints {"ms": [...]}."""
    from oracle import RefTree
    pts = make_points_checker(a.n, a.dist, a.seed)
    ref = RefTree()
    cores = a.ref_threads or ref.hardware_threads()
    ms = ref.time(pts, cores, a.ref_iters)
    print(json.dumps({"ms": [float(x) for x in ms], "cores": cores}), flush=True)
    return 0


def ref_time_isolated(a, seed, iters):
    """Wall ms of `iters` runs of the reference's own CPU pipeline (oracle/_ref)
    on the cloud make_points_checker(n, dist, seed) gives, in a child process: the
    reference's stage 7 writes out of bounds on some clouds (negative octree
    offsets reach func_octree.hpp:101), which must not take this process down.
    Returns (ms list, cores) or (None, reason)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--ref-time-child", "--n", str(a.n),
           "--dist", a.dist, "--seed", str(seed), "--ref-iters", str(iters)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
    except subprocess.TimeoutExpired:
        return None, "the reference's CPU path did not finish in 30 minutes"
    if r.returncode != 0:
        how = f"signal {-r.returncode}" if r.returncode < 0 else f"exit {r.returncode}"
        return None, (f"the reference's CPU path ended with {how} on this cloud "
                      f"(out-of-bounds writes in its stage 7)")
    out = json.loads(r.stdout.strip().splitlines()[-1])
    return out["ms"], out["cores"]


def ref_cuda_child(a):
    """Child side of ref_cuda_isolated: the same cloud through the
    reference's own CUDA stages 1-7 (oracle/_ref/libref_tree_cuda.so)."""
    from oracle import RefTreeCuda
    pts = make_points_checker(a.n, a.dist, a.seed)
    out = RefTreeCuda().time(pts, a.ref_iters)
    print(json.dumps(out), flush=True)
    return 0


def ref_cuda_isolated(a, warmup=2, iters=10):
    """The reference's CUDA path (cuda::run_stage1..7, pipe_main_baseline.cpp:
    55-92, compiled for sm_100a) on this workload's cloud, in a child process
    on the same GPU: median wall ms per run of its seven synchronous stages.
    32-bit keys and sizes that are multiples of 1024 only (its k_FindDups
    reads whole 1,024-key tiles).  A comparison point, not a parity check:
    the driver copies the sorted keys into the buffer its stage 3 reads (the
    buffer contract its dispatcher does not honour) and runs its stage 4 and
    stage 7 only after device-side checks of their inputs."""
    from oracle import ref_cuda_available
    if a.key_bits != 32 or a.n % 1024 or not ref_cuda_available():
        return {"unavailable": "32-bit keys, n a multiple of 1024 and oracle/_ref built only"}
    cmd = [sys.executable, os.path.abspath(__file__), "--ref-cuda-child", "--n", str(a.n),
           "--dist", a.dist, "--seed", str(a.seed), "--ref-iters", str(warmup + iters)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    except subprocess.TimeoutExpired:
        return {"unavailable": "the reference's CUDA path did not finish in 10 minutes"}
    if r.returncode != 0:
        return {"unavailable": f"the reference's CUDA path exited with {r.returncode}: "
                               f"{r.stderr.strip()[-300:]}"}
    out = json.loads(r.stdout.strip().splitlines()[-1])
    ms = out.pop("ms")[warmup:]
    t = statistics.median(ms)
    if out.get("all_stages_ran"):
        out.update({"ms_per_step": round(t, 4), "value": a.n / (t / 1e3), "unit": "points/s",
                    "sample": f"median of {iters} runs after {warmup} warm-up runs, wall time "
                              f"of its seven synchronous stages (device-side checks excluded)"})
    else:
        ran = [k + 1 for k, x in enumerate(out["stage_ms_last_run"]) if x > 0]
        out.update({"value": None, "stages_run": ran, "ms_stages_run": round(t, 4),
                    "sample": f"median of {iters} runs after {warmup} warm-up runs, wall time "
                              f"of the stages that ran ({ran}; device-side checks excluded)"})
    return out


def copy_floor_ms(app, h_pts, outs, m, reps):
    """Device time of one step's host copies alone: the points host to device
    on one stream while the five octree arrays (m rows) go device to host on
    another, from and to the same pinned buffers the end-to-end step uses."""
    import torch
    pairs = [(outs["children"][:m], app.oct_children[:m]), (outs["corner"][:m], app.oct_corner[:m]),
             (outs["cell_size"][:m], app.oct_cell_size[:m]),
             (outs["child_node_mask"][:m], app.oct_child_node_mask[:m]),
             (outs["child_leaf_mask"][:m], app.oct_child_leaf_mask[:m])]
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

    def step():
        with torch.cuda.stream(s_in):
            app.u_input_points.copy_(h_pts, non_blocking=True)
        with torch.cuda.stream(s_out):
            for h, d in pairs:
                h.copy_(d, non_blocking=True)

    cur = torch.cuda.current_stream()
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(cur)
    s_in.wait_stream(cur)
    s_out.wait_stream(cur)
    for _ in range(reps):
        step()
    cur.wait_stream(s_in)
    cur.wait_stream(s_out)
    e1.record(cur)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def rank_barrier(world):
    """Every rank waits for the others (the timed regions start and end
    together); nothing with one process."""
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def rank_max(x, world, device):
    """The largest of every rank's x (each rank's step time: the job's time is
    its slowest rank's), the same value on every rank."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def port_time(pts, a, iters):
    from oracle import Oracle
    orc = Oracle()
    ms = []
    for _ in range(iters):
        t0 = time.perf_counter()
        orc.run(pts, key_bits=a.key_bits)
        ms.append((time.perf_counter() - t0) * 1e3)
    return ms


def cpu_baseline(rw, pts, a):
    from oracle import ref_available
    note = None
    if a.key_bits == 32 and ref_available():
        first, info = ref_time_isolated(a, a.seed, 1)
        if first is not None:
            iters = int(min(10, max(3, 15000.0 / max(first[0], 1.0))))
            ms, info = ref_time_isolated(a, a.seed, iters)
            if ms is not None:
                t = statistics.median(ms)
                return {"value": a.n / (t / 1e3), "unit": "points/s", "cores": info,
                        "kind": "reference",
                        "sample": f"median of {iters} runs of cpu::run_stage1..7 (verbatim, "
                                  f"{info} threads) on the same n={a.n} cloud, after 1 warm "
                                  f"run"}
        note = info  # why the reference could not be timed
    t = port_time(pts, a, 1)[0]
    line = {"value": a.n / (t / 1e3), "unit": "points/s", "cores": 1, "kind": "port",
            "sample": f"1 run of the C restatement on the n={a.n} cloud"}
    if note:
        line["note"] = note
    return line


def main():
    a = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.ref_time_child:
        return ref_time_child(a)
    if a.ref_cuda_child:
        return ref_cuda_child(a)
    if a.impl == "reference":
        return run_reference(a, rank)

    import torch
    import torch.distributed as dist
    from __graft_entry__ import _load_package

    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    rw = _load_package()
    K = 4 if a.key_bits == 32 else 8

    pts = make_points(rw, a.n, a.dist, a.seed + rank)
    app = rw.AppData(a.n, a.key_bits, points=pts)
    im = rw.ImStorage(a.n, a.key_bits, a.radix_bits)
    if a.sort_variant >= 0:
        im.set_sort_variant(a.sort_variant)
    passes = sort_passes(a)

    def barrier():
        rank_barrier(world)

    def max_over_ranks(x):
        return rank_max(x, world, "cuda")

    stream = torch.cuda.current_stream()
    for _ in range(a.warmup):
        rw.run_pipeline(app, im)
    u, m = app.get_n_unique(), app.get_n_octree_nodes()

    mismatches = None
    if not a.no_verify and rank == 0:
        from oracle import Oracle
        want = Oracle().run(pts, key_bits=a.key_bits).trimmed()
        got = app.results()
        mismatches = sum(
            1 for k, v in want.items()
            if (np.ascontiguousarray(got[k]).tobytes() != np.ascontiguousarray(v).tobytes()
                if isinstance(v, np.ndarray) else got[k] != v))

    # ---- device-resident timed region ------------------------------------
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        ev0.record(stream)
        for _ in range(a.steps):
            rw.pipeline_enqueue(app, im)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    rw.pipeline_finish(app, im)
    ms_step = max_over_ranks(ev0.elapsed_time(ev1) / a.steps)
    value = a.n * world / (ms_step / 1e3)
    if a.only_device:
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "points/s",
                              "ms_per_step": ms_step, "only_device": True,
                              "mismatches_vs_oracle": mismatches}), flush=True)
        return 0

    # ---- several clouds in flight --------------------------------------------
    # More AppData / scratch pairs, each on its own stream, the K timed steps
    # taken by the pairs in turn (the same cloud, the same seven stages each
    # step): one cloud's kernels with few blocks (the one-block tile scans, the
    # sort set-up, the octree's far links) and every kernel's ramp-up and tail
    # then overlap another cloud's kernels, as consecutive clouds of a stream of
    # clouds can.  `value` is this throughput; `one_stream` is the region
    # above, one cloud after another on one stream.
    one_stream_ms = ms_step
    inflight = max(1, a.slots)
    extra = []
    for _ in range(inflight - 1):
        app_k = rw.AppData(a.n, a.key_bits, points=pts)
        im_k = rw.ImStorage(a.n, a.key_bits, a.radix_bits)
        if a.sort_variant >= 0:
            im_k.set_sort_variant(a.sort_variant)
        extra.append((app_k, im_k, torch.cuda.Stream()))
    for app_k, im_k, s_k in extra:
        for _ in range(a.warmup):
            rw.run_pipeline(app_k, im_k, s_k)
    torch.cuda.synchronize()
    slot_mismatches = None
    if mismatches is not None:
        slot_mismatches = 0
        for app_k, _, _ in extra:
            got_k = app_k.results()
            slot_mismatches += sum(
                1 for k, v in want.items()
                if (np.ascontiguousarray(got_k[k]).tobytes() != np.ascontiguousarray(v).tobytes()
                    if isinstance(v, np.ndarray) else got_k[k] != v))
    pairs = [(app, im, stream)] + extra
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks_k:
        ev2.record(stream)
        for _, _, s_k in extra:
            s_k.wait_stream(stream)
        for i in range(a.steps):
            app_k, im_k, s_k = pairs[i % inflight]
            rw.pipeline_enqueue(app_k, im_k, s_k)
        for _, _, s_k in extra:
            stream.wait_stream(s_k)
        ev3.record(stream)
        torch.cuda.synchronize()
    barrier()
    for app_k, im_k, s_k in pairs:
        rw.pipeline_finish(app_k, im_k, s_k)
    ms_step = max_over_ranks(ev2.elapsed_time(ev3) / a.steps)
    value = a.n * world / (ms_step / 1e3)
    one_stream = {"value": a.n * world / (one_stream_ms / 1e3), "ms_per_step": one_stream_ms,
                  "clocks": clocks.summary()}
    clocks = clocks_k
    del extra, pairs

    # ---- per-kernel device times inside the pipeline -----------------------
    kms = rw.profile_pipeline(app, im, reps=max(3, min(10, a.steps)))
    hbm, peak_kind = peaks()
    stages = {}
    for name, t in kms.items():
        by = kernel_bytes(name, a.n, u, m, K)
        gbs = by / (t * 1e-3) / 1e9 if t > 0 and by else None
        stages[name] = {"ms": round(t, 5), "bytes": by,
                        "gbs": round(gbs, 1) if gbs else None,
                        "frac": round(gbs / hbm, 3) if gbs else None}
    dom = max(kms, key=kms.get)
    tt = traffic_table().get("entries", {})
    dom_traffic = None
    key = f"{a.dist}-{a.key_bits}-{dom}"
    if key in tt and a.n == 1 << 24:  # captured at this size (profiles/ncu_traffic.json)
        dom_traffic = tt[key]["traffic"]
    dom_gbs = stages[dom]["gbs"]
    roofline = {"bound": "hbm", "kernel": dom, "achieved": dom_gbs, "peak": hbm,
                "unit": "GB/s", "frac": round(dom_gbs / hbm, 4) if dom_gbs else None,
                "traffic": dom_traffic, "peak_source": f"{peak_kind} hbm_gbs"}
    pipe_b = pipeline_bytes(a.n, u, m, K, passes)
    pipe_gbs = pipe_b / (ms_step * 1e-3) / 1e9

    # ---- end to end through the host-facing C ABI call ---------------------
    h_pts = torch.from_numpy(pts).pin_memory()
    cap = rw.octree_capacity(a.n)
    outs = {
        "children": torch.empty((cap, 8), dtype=torch.int32).pin_memory(),
        "corner": torch.empty((cap, 4), dtype=torch.float32).pin_memory(),
        "cell_size": torch.empty(cap, dtype=torch.float32).pin_memory(),
        "child_node_mask": torch.empty(cap, dtype=torch.int32).pin_memory(),
        "child_leaf_mask": torch.empty(cap, dtype=torch.int32).pin_memory(),
    }
    outs_np = {k: v.numpy() for k, v in outs.items()}
    h_np = h_pts.numpy()
    e2e_steps = max(3, min(a.steps, 10))
    # one slot: rw_tree_run_host (copy in, pipeline, copy out, wait) per step
    for _ in range(2):
        rw.run_host(app, im, h_np, outs_np)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(e2e_steps):
        rw.run_host(app, im, h_np, outs_np)
    e1.record(stream)
    torch.cuda.synchronize()
    single_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps)
    # three slots on three streams: submit(k) then collect(k-2).  A slot's
    # stream runs copy in, pipeline, copy out in order; with three slots the
    # copy in of cloud k does not wait behind the copy out of the cloud before
    # it on the same stream while another cloud's copy out holds the
    # device-to-host direction
    n_slots = max(2, a.e2e_slots)
    slots = [(app, im, torch.cuda.Stream(), outs_np)]
    for _ in range(n_slots - 1):
        ax = rw.AppData(a.n, a.key_bits, points=pts)
        ix = rw.ImStorage(a.n, a.key_bits, a.radix_bits)
        if a.sort_variant >= 0:
            ix.set_sort_variant(a.sort_variant)
        slots.append((ax, ix, torch.cuda.Stream(),
                      {k: torch.empty_like(v).pin_memory().numpy() for k, v in outs.items()}))

    def streamed(k_steps):
        lag = n_slots - 1
        for k in range(k_steps + lag):
            if k < k_steps:
                cur = slots[k % n_slots]
                rw.host_submit(cur[0], cur[1], h_np, cur[2])
            if k >= lag:
                prev = slots[(k - lag) % n_slots]
                rw.host_collect(prev[0], prev[1], prev[3], prev[2])

    streamed(4)
    torch.cuda.synchronize()
    barrier()
    s0 = slots[0][2]
    e0.record(s0)
    for sl in slots[1:]:
        sl[2].wait_event(e0)
    streamed(e2e_steps)
    for sl in slots[1:]:
        s0.wait_stream(sl[2])
    e1.record(s0)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps)
    m2 = app.get_n_octree_nodes()
    d2h = 60 * m2 + 16
    floor_ms = copy_floor_ms(app, h_pts, outs, m2, e2e_steps)
    e2e = {"value": a.n * world / (e2e_ms / 1e3), "unit": "points/s",
           "h2d_bytes_per_step": 16 * a.n, "d2h_bytes_per_step": d2h,
           "ms_per_step": round(e2e_ms, 4),
           "single_slot_ms_per_step": round(single_ms, 4),
           "copy_floor_ms": round(floor_ms, 4),
           "copy_floor_note": "the same step's copies alone (points host to device on one "
                              "stream, the five octree arrays device to host on another, "
                              "pinned buffers, no kernels), the PCIe bound of this number",
           "path": f"rw_tree_host_submit / rw_tree_host_collect on {n_slots} AppData/scratch "
                   f"pairs and {n_slots} streams: pinned host points -> H2D -> 7 stages -> "
                   "counts + octree rows (children, corner, cell_size, masks) D2H, every step"}
    del slots[1:]

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(rw, pts, a)
    ref_cuda = None
    if rank == 0 and world == 1 and not a.no_ref_cuda:
        ref_cuda = ref_cuda_isolated(a)
        if ref_cuda.get("stages_run"):
            # our device time of the same stages (4 and 5 are one fused kernel here)
            ours = ["morton_histogram", "sort_init"] + [f"sort_pass{p}" for p in range(passes)] + \
                ["unique", "radix_tree_edges"]
            if ref_cuda["stages_run"] == [1, 2, 3, 4, 5]:
                ref_cuda["ours_ms_stages_1_5"] = round(sum(kms[k] for k in ours if k in kms), 4)

    forms = None
    if rank == 0 and not a.no_forms:
        del app, im
        torch.cuda.empty_cache()
        forms = {"batched": measure_batch(rw, a)}
        torch.cuda.empty_cache()
        forms["learned"] = measure_learned(rw, a)
        torch.cuda.empty_cache()
        forms["combined"] = measure_combined(rw, a)

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": f"u{a.key_bits}", "data": "synthetic",
        "config": config_of(a),
        "n_unique": u, "n_octree_nodes": m, "mismatches_vs_oracle": mismatches,
        "slots": inflight, "other_slots_mismatches_vs_oracle": slot_mismatches,
        "one_stream": one_stream,
        "pipeline_roofline": {"bytes_per_step": pipe_b, "achieved_gbs": round(pipe_gbs, 1),
                              "frac": round(pipe_gbs / hbm, 4)},
        "roofline": roofline, "stages": stages, "e2e": e2e, "cpu_baseline": cpu,
        "reference_cuda": ref_cuda,
        # the fused pipeline's own kernels per step: keys, sort set-up, P passes,
        # unique (3), radix tree, edge sums (2), octree (2); the scratch memset
        # and the status copy are not kernels of this library
        "clocks": clocks.summary(), "gpu_launches": (10 + passes) * a.steps,
        "forms": forms,
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
