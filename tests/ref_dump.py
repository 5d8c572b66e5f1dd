"""Run the reference (oracle/_ref/libatjup_ref.so) in a child process and dump its state.

    python tests/ref_dump.py OUT.npz [--iters N] [--rk4] [--moist] [--threads T]

Writes the reference's dry initial state (species zeroed unless --moist), its grid, its model
constants, and -- with --iters N -- the state after N iterations of the harness loop
(cJupiterModel.cpp:1032-1381 schedule), or with --rk4 the state after one RungeKuttaJup.
Test infrastructure only.
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from oracle_bridge import DRY_ENV, DYN_FIELDS, Reference  # noqa: E402

CONSTS = ("dt", "re", "pr", "g", "omega", "u_0", "t_ref", "L_atm", "r_mix", "R_mix", "cp_mix",
          "Coriolis", "centrifugal", "buoyancy")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out")
    ap.add_argument("--iters", type=int, default=0)
    ap.add_argument("--rk4", action="store_true")
    ap.add_argument("--pressure", action="store_true")
    ap.add_argument("--moist", action="store_true")
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args()
    out_dir = tempfile.mkdtemp(prefix="atjup_ref_")
    ref = Reference(dict(DRY_ENV), out_dir + "/run", threads=a.threads, zero_species=not a.moist)
    data = {}
    g = ref.grid()
    for k, v in g.items():
        data["grid_" + k] = v
    for n, v in ref.fields().items():
        data["in_" + n] = v
    for c in CONSTS:
        data["const_" + c] = np.array(ref.scalar(c))
    if a.rk4:
        ref.quiet(ref.L.ref_rk4)
        for n in DYN_FIELDS:
            data["out_" + n] = ref.get(n)
        data["out_buoy_ref"] = ref.get1("buoy_ref_level")
    elif a.pressure:
        ref.quiet(ref.L.ref_pressure)
        for n in ("p_dyn", "aux_u", "aux_v", "aux_w"):
            data["out_" + n] = ref.get(n)
    elif a.iters > 0:
        for it in range(1, a.iters + 1):
            rc = ref.quiet(ref.L.ref_iteration, it, 1 if it == 1 else 0, 0 if a.moist else 1)
            if rc != 0:
                raise SystemExit(f"ref_iteration rc={rc}")
        for n in DYN_FIELDS:
            data["out_" + n] = ref.get(n)
    np.savez(a.out, **data)
    sys.stdout.flush()
    os._exit(0)   # the reference's destructor is not needed; skip interpreter teardown


if __name__ == "__main__":
    main()
