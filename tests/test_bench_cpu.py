"""bench.py's CPU-side contract: the reference arm's JSON line, and the child
process that times the reference's own CPU pipeline (which must not take the
bench down when that pipeline crashes on a cloud)."""
import importlib.util
import json
import os
import subprocess
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", BENCH)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def args(**kw):
    base = dict(n=20000, dist="uniform", key_bits=32, seed=20260101, steps=2, warmup=1,
                gpus=1, ref_threads=0, ref_iters=1)
    base.update(kw)
    return types.SimpleNamespace(**base)


def test_reference_arm_line():
    """`bench.py --impl reference` prints one JSON line with the fields the
    driver reads (value, unit, cpu_baseline, e2e with zero copy bytes)."""
    r = subprocess.run([sys.executable, BENCH, "--impl", "reference", "--n", "20000",
                        "--steps", "2", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "points/s" and line["higher_is_better"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_reference_timed_in_a_child():
    bench = load_bench()
    from oracle import ref_available
    if not ref_available():
        pytest.skip("the reference's CPU library is not built here")
    ms, cores = bench.ref_time_isolated(args(), 20260101, 2)
    assert ms is not None, cores
    assert len(ms) == 2 and all(t > 0 for t in ms) and cores >= 1


def test_reference_child_failure_is_reported(monkeypatch):
    """A child that dies (here: an interpreter that exits with an error) gives
    (None, reason) instead of an exception."""
    bench = load_bench()
    monkeypatch.setattr(bench.sys, "executable", "/bin/false")
    ms, why = bench.ref_time_isolated(args(), 20260101, 1)
    assert ms is None and "exit 1" in why


def test_reference_arm_loads_no_product_library():
    """The reference arm builds its cloud from the oracle's generators and
    times the reference's own code: librw_tree.so is never mapped, and its
    config object is the one our arm prints."""
    code = (
        "import sys, json, types; sys.argv=['bench.py'];"
        "import importlib.util as u;"
        f"spec=u.spec_from_file_location('b', {BENCH!r}); b=u.module_from_spec(spec);"
        "spec.loader.exec_module(b);"
        "a=types.SimpleNamespace(n=20000, dist='uniform', key_bits=32, radix_bits=0,"
        " seed=20260101, steps=2, warmup=1, gpus=1, ref_threads=0, ref_iters=1);"
        "b.run_reference(a, 0);"
        "maps=open('/proc/self/maps').read();"
        "print(json.dumps({'product_mapped': 'librw_tree' in maps,"
        " 'config': b.config_of(a)}))")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.strip().splitlines()]
    ref_line, probe = lines[0], lines[-1]
    assert probe["product_mapped"] is False
    assert ref_line["config"] == probe["config"]
    assert set(probe["config"]) >= {"workload", "n_points", "key_bits", "radix_bits",
                                    "sort_passes", "parallelism"}


def _two_rank_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bench = load_bench()
    bench.rank_barrier(world)
    step_ms = [1.5, 4.25][rank]  # each rank's own step time
    out[rank] = bench.rank_max(step_ms, world, "cpu")
    bench.rank_barrier(world)
    dist.destroy_process_group()


def test_two_ranks_take_the_slowest_step():
    """The replicas-only multi-GPU path: with world size 2 (gloo, CPU) both
    ranks pass the barriers and agree on the slowest rank's step time, which
    bench.py divides the whole job's points by."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_two_rank_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 4.25


def test_clock_sampler_reads_nvml_inside_the_region(monkeypatch):
    """The clock sampler takes NVML samples from a thread while the timed region
    runs (read-only queries: clock, max clock, clock-event reasons) and reports
    the median, the sample count and every throttle reason seen.  A fake NVML
    module stands in for the driver; a region with a power-capped sample
    reports sw_power_cap."""
    import time

    state = {"calls": 0, "shut": False}

    class FakeNvml(types.ModuleType):
        NVML_CLOCK_SM = 1

        def nvmlInit(self):
            pass

        def nvmlShutdown(self):
            state["shut"] = True

        def nvmlDeviceGetHandleByPciBusId(self, bus):
            raise RuntimeError("no PCI address here")

        def nvmlDeviceGetHandleByIndex(self, i):
            return ("dev", i)

        def nvmlDeviceGetMaxClockInfo(self, h, kind):
            return 1965

        def nvmlDeviceGetClockInfo(self, h, kind):
            state["calls"] += 1
            return 1965 if state["calls"] % 2 else 1950

        def nvmlDeviceGetCurrentClocksEventReasons(self, h):
            return 0x4 if state["calls"] == 3 else 0

    monkeypatch.setitem(sys.modules, "pynvml", FakeNvml("pynvml"))
    bench = load_bench()
    with bench.ClockSampler(0, period_s=0.001) as c:
        time.sleep(0.05)
    s = c.summary()
    assert state["shut"]
    assert s["samples"] >= 5 and s["samples"] == state["calls"]
    assert s["sm_max_mhz"] == 1965.0 and s["sm_mhz"] in (1950.0, 1957.5, 1965.0)
    assert s["reasons"] == ["sw_power_cap"]
    assert "nvml" in s["source"] and "index" in s["source"]
