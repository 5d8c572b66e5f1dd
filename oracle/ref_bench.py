"""Time the reference's own CPU implementation of one model iteration (dry or full physics).

TEST AND CPU-BASELINE INFRASTRUCTURE: used only by bench.py's CPU legs (the reference arm and the
cpu_baseline figure). Runs oracle/_ref/libatjup_ref.so -- the unmodified reference built from its
sources -- in this process: the reference's initialisation with the benchmark configuration's
seeded initial state applied (oracle/baseline_state.py; untimed), `warmup` iterations (untimed),
then `steps` iterations of the cJupiterModel.cpp:1032-1381 schedule -- the dry configuration, or
with --phys the reference's default full physics (the k-omega SST closure, radiation,
precipitation, the saturation adjustments, the NH4SH equilibrium, the chemistry block and the
moist convective adjustment every iteration, as baseline_state.PHYS_ENV sets), both with the
projection around the obstacle every 10 iterations (the reference's default) -- each timed by
wall clock on the host. Prints one JSON line.

    python oracle/ref_bench.py --steps K --warmup W [--threads T] [--phys]
    python oracle/ref_bench.py --cone N [--threads T]

With --cone N: no iterations; N in-loop projections around the obstacle
(projectAroundObstacle(true), InitValues_Jup.cpp:1595-1822) on the dry configuration's state, the
first from zero and the rest warm-started, each timed by wall clock.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
LIB = HERE / "_ref" / "libatjup_ref.so"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--phys", action="store_true")
    ap.add_argument("--cone", type=int, default=0)
    a = ap.parse_args()
    if not LIB.exists():
        print(json.dumps({"unavailable": f"{LIB} not built"}))
        return
    import baseline_state as BS
    config = "phys" if a.phys else "dry"
    threads = a.threads or os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    out_dir = tempfile.mkdtemp(prefix="atjup_refbench_")
    t0 = time.perf_counter()
    try:
        ref = BS.make(config, out_dir + "/run", threads=threads)
    except Exception as e:   # noqa: BLE001 -- reported as the arm's unavailability
        print(json.dumps({"unavailable": f"reference initialisation failed: {e}"}))
        return
    t_init = time.perf_counter() - t0
    L = ref.L
    if a.cone:
        times = []
        L.ref_quiet(1)
        for _ in range(a.cone):
            t0 = time.perf_counter()
            L.ref_cone_proj(0)
            times.append(time.perf_counter() - t0)
        L.ref_quiet(0)
        print(json.dumps({"cone_s_per_call": sum(times) / len(times), "call_times": times,
                          "threads": threads, "state": BS.describe(config)}))
        sys.stdout.flush()
        os._exit(0)
    times = []
    rc = 0
    L.ref_quiet(1)
    for it in range(1, a.warmup + a.steps + 1):
        t0 = time.perf_counter()
        rc = L.ref_iteration(it, 1 if it == 1 else 0, 0 if a.phys else 1)
        dt = time.perf_counter() - t0
        if rc != 0:
            break
        if it > a.warmup:
            times.append(dt)
    L.ref_quiet(0)
    if rc != 0:
        print(json.dumps({"unavailable": f"ref_iteration rc={rc}"}))
    else:
        print(json.dumps({"s_per_step": sum(times) / len(times), "steps": len(times),
                          "step_times": times, "threads": threads, "init_s": t_init,
                          "state": BS.describe(config)}))
    sys.stdout.flush()
    os._exit(0)


if __name__ == "__main__":
    main()
