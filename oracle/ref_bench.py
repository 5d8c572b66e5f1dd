"""Time the reference's own CPU implementation of one model iteration (dry or full physics).

TEST AND CPU-BASELINE INFRASTRUCTURE: used only by bench.py's CPU legs (the reference arm and the
cpu_baseline figure). Runs oracle/_ref/libatjup_ref.so -- the unmodified reference built from its
sources -- in this process: the reference's initialisation (untimed), `warmup` iterations
(untimed), then `steps` iterations of the cJupiterModel.cpp:1032-1381 schedule -- the dry
configuration, or with --phys the full physics (the closure, radiation, precipitation, the
saturation adjustments, the NH4SH equilibrium and the chemistry block on; moist convective
adjustment off) -- each timed by wall clock on the host. Prints one JSON line.

    python oracle/ref_bench.py --steps K --warmup W [--threads T] [--phys]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import tempfile
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libatjup_ref.so"

DRY_ENV = {
    "ATJUP_NO_SEAMOUNT": "0", "ATJUP_PRECIP": "0", "ATJUP_RADIATION": "0", "ATJUP_TURB": "0",
    "ATJUP_MCA": "0", "ATJUP_NH4SH_EQ": "0", "ATJUP_CONE_PROJ_STRIDE": "0",
    "ATJUP_VEL_SHAPIRO_ORDER": "4", "ATJUP_VEL_SHAPIRO_INLOOP": "1",
    "ATJUP_RESTART_STRIDE": "0", "ATJUP_VTK_STRIDE": "100000", "ATJUP_PANORAMA_STRIDE": "100000",
}


# the reference's default full physics: closure, radiation, precipitation, NH4SH equilibrium and
# the moist convective adjustment every iteration
PHYS_ENV = {**DRY_ENV, "ATJUP_TURB": "1", "ATJUP_PRECIP": "1", "ATJUP_RADIATION": "1",
            "ATJUP_NH4SH_EQ": "1", "ATJUP_MCA": "1"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--phys", action="store_true")
    a = ap.parse_args()
    if not LIB.exists():
        print(json.dumps({"unavailable": f"{LIB} not built"}))
        return
    os.environ.update(PHYS_ENV if a.phys else DRY_ENV)
    threads = a.threads or os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    L = ctypes.CDLL(str(LIB))
    out_dir = tempfile.mkdtemp(prefix="atjup_refbench_")
    L.ref_quiet(1)
    t0 = time.perf_counter()
    rc = L.ref_create((out_dir + "/run").encode(), threads)
    t_init = time.perf_counter() - t0
    if rc != 0:
        L.ref_quiet(0)
        print(json.dumps({"unavailable": f"ref_create rc={rc}"}))
        return
    times = []
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
                          "step_times": times, "threads": threads, "init_s": t_init}))
    sys.stdout.flush()
    os._exit(0)


if __name__ == "__main__":
    main()
