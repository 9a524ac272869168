"""Autotuner of the batched pipeline's sort.

For each size class of clouds it times every onesweep variant of the menu
(threads per CTA, keys per thread, warp ranking scheme) on a synthetic batch of
that class, for each digit width (8, 10 and 11 bits), and keeps the fastest.  The
digit width is one per batch (the digit histograms of every pass are built
while the keys are encoded), so the width with the smallest summed time wins
and each class gets its best variant at that width.

The table it writes (JSON) is what ``Batch(..., tuning=...)`` applies through
``rw_tree_batch_set_classes``.  Run on the target GPU:

    python redwood-comp_b200/autotune.py --key-bits 32 --out table.json
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TUNING_DIR = os.path.join(HERE, "tuning")

# class upper bounds (points per cloud); the last class is unbounded
DEFAULT_BOUNDS = (16384, 131072)
CLOUD_RANGE = (1024, 262144)


def synth_clouds(rw, lo: int, hi: int, total_points: int, seed: int):
    """Clouds with sizes log-uniform in [lo, hi], uniform or Gaussian mixture
    by seed, until `total_points` is reached."""
    rng = np.random.default_rng(seed)
    clouds, total, c = [], 0, 0
    while total < total_points:
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        if rng.random() < 0.5:
            pts = rw.generate_points(n, rw.GEN_UNIFORM, seed * 100003 + c)
        else:
            pts = rw.generate_points(n, rw.GEN_GAUSSIAN_MIXTURE, seed * 100003 + c,
                                     n_components=int(rng.integers(8, 65)))
        clouds.append(pts)
        total += n
        c += 1
    return clouds


def time_batch(batch, reps: int) -> float:
    import torch
    for _ in range(2):
        batch.run(graph=True)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(reps):
        batch.enqueue(graph=True)
    e1.record(s)
    batch.finish()
    return e0.elapsed_time(e1) / reps


def tune(rw, key_bits: int = 32, bounds=DEFAULT_BOUNDS, digit_widths=(8, 10, 11),
         points_per_class: int = 6_000_000, reps: int = 5, seed: int = 1, log=print) -> dict:
    lows = [CLOUD_RANGE[0]] + [b + 1 for b in bounds]
    highs = list(bounds) + [CLOUD_RANGE[1]]
    menu = rw.sort_variants()
    measured = {}
    for d in digit_widths:
        per_class = []
        for k, (lo, hi) in enumerate(zip(lows, highs)):
            clouds = synth_clouds(rw, lo, hi, points_per_class, seed + 17 * k)
            batch = rw.Batch(clouds, key_bits, radix_bits=d, octree_ratio=1.5)
            times = {}
            for v in menu:
                if v["key_bits"] != key_bits or v["radix_bits"] != d:
                    continue
                batch.set_sort_variant(v["index"])
                times[v["index"]] = time_batch(batch, reps)
                log(f"key_bits={key_bits} digits={d} class={k} [{lo},{hi}] "
                    f"variant={v['index']} ({v['threads']}x{v['keys_per_thread']} "
                    f"rank={v['rank']}): {times[v['index']]:.4f} ms")
            best = min(times, key=times.get)
            per_class.append({"min_points": lo, "max_points": hi, "variant": best,
                              "ms_per_run": times[best], "points": int(sum(c.shape[0] for c in clouds)),
                              "all_ms": times})
            batch.close()
        measured[d] = per_class
    best_d = min(measured, key=lambda d: sum(c["ms_per_run"] for c in measured[d]))
    classes = []
    for c in measured[best_d]:
        v = menu[c["variant"]]
        classes.append({"max_points": c["max_points"], "variant": c["variant"],
                        "threads": v["threads"], "keys_per_thread": v["keys_per_thread"],
                        "rank": v["rank"], "ms_per_run": round(c["ms_per_run"], 5)})
    import torch
    return {
        "gpu": torch.cuda.get_device_name(0),
        "key_bits": key_bits,
        "radix_bits": best_d,
        "classes": classes,
        "measured_ms": {str(d): [round(c["ms_per_run"], 5) for c in measured[d]] for d in measured},
        "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
    }


def table_path(key_bits: int) -> str:
    return os.path.join(TUNING_DIR, f"b200_u{key_bits}.json")


def load_table(key_bits: int) -> dict | None:
    try:
        with open(table_path(key_bits)) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def resolve_variant(entry: dict, key_bits: int, radix_bits: int, menu: list) -> int | None:
    """Index in the current menu of the variant a table entry describes
    (threads, keys per thread, ranking), or None when the menu lacks it.
    Tables name variants by shape, so that adding menu entries does not
    invalidate them."""
    for v in menu:
        if (v["key_bits"], v["radix_bits"], v["threads"], v["keys_per_thread"], v["rank"]) == \
                (key_bits, radix_bits, int(entry["threads"]), int(entry["keys_per_thread"]),
                 int(entry["rank"])):
            return v["index"]
    return None


def class_list(table: dict, menu: list) -> list | None:
    """[(max_points, variant index)] for Batch.set_classes, or None when a
    class's variant is no longer in the menu."""
    out = []
    for c in table["classes"]:
        idx = resolve_variant(c, int(table["key_bits"]), int(table["radix_bits"]), menu)
        if idx is None:
            return None
        out.append((int(c["max_points"]), idx))
    return out


def main(argv=None) -> int:
    import argparse
    sys.path.insert(0, os.path.dirname(HERE))
    from __graft_entry__ import _load_package
    p = argparse.ArgumentParser()
    p.add_argument("--key-bits", type=int, default=32, choices=(32, 64))
    p.add_argument("--out", default=None)
    p.add_argument("--points-per-class", type=int, default=6_000_000)
    p.add_argument("--reps", type=int, default=5)
    a = p.parse_args(argv)
    rw = _load_package()
    table = tune(rw, a.key_bits, points_per_class=a.points_per_class, reps=a.reps)
    out = a.out or table_path(a.key_bits)
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    with open(out, "w") as f:
        json.dump(table, f, indent=1)
    print(json.dumps({k: v for k, v in table.items() if k != "measured_ms"}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
